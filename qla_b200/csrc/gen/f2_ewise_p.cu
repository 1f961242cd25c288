// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F2 ewise_p entry points (extern "C"), reference: lib/perl/build_qla.pl:403-469, 1256-1420 (element-wise families)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_F2_P_veq_c_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_c_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_r_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_r_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_c_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_c_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_r_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_r_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_c_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_c_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_r_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_r_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_c_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_c_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_r_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_r_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_C_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_C_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_C_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_C_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_C_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_C_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_C_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_C_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pC_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pC_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pC_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pC_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pC_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pC_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pC_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pC_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_Ca_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_Ca_times_P");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_Ca_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_Ca_times_pP");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_Ca_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_Ca_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_Ca_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_Ca_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pCa_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pCa_times_P");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pCa_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pCa_times_pP");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pCa_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pCa_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pCa_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pCa_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_R_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_R_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_R_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_R_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_R_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_R_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_R_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_R_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pR_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pR_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pR_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pR_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pR_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pR_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pR_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pR_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_conj_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_veq_conj_P");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_conj_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_veq_conj_pP");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_i_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_veq_i_P");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_i_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_veq_i_pP");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_veq_Pa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pPa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_transpose_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_veq_transpose_P");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_transpose_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_veq_transpose_pP");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_veq_P");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pP");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_c_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_c_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_r_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_r_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_c_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_c_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_r_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_r_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_c_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_c_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_r_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_r_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_c_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_c_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_r_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_r_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_C_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_C_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_C_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_C_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_C_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_C_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_C_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_C_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_pC_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_pC_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_pC_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_pC_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_pC_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_pC_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_pC_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_pC_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_Ca_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_Ca_times_P");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_Ca_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_Ca_times_pP");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_Ca_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_Ca_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_Ca_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_Ca_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_pCa_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_pCa_times_P");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_pCa_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_pCa_times_pP");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_pCa_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_pCa_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_pCa_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_pCa_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_R_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_R_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_R_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_R_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_R_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_R_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_R_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_R_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_pR_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_pR_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_pR_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_pR_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_pR_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_pR_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_pR_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_pR_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_conj_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_conj_P");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_conj_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_conj_pP");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_i_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_i_P");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_i_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_i_pP");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_Pa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_pPa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_transpose_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_transpose_P");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_transpose_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_transpose_pP");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_P");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_pP");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_c_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_c_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_r_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_r_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_c_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_c_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_r_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_r_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_c_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_c_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_r_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_r_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_c_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_c_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_r_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_r_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_C_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_C_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_C_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_C_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_C_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_C_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_C_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_C_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_pC_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_pC_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_pC_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_pC_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_pC_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_pC_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_pC_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_pC_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_Ca_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_Ca_times_P");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_Ca_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_Ca_times_pP");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_Ca_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_Ca_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_Ca_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_Ca_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_pCa_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_pCa_times_P");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_pCa_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_pCa_times_pP");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_pCa_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_pCa_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_pCa_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_pCa_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_R_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_R_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_R_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_R_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_R_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_R_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_R_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_R_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_pR_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_pR_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_pR_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_pR_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_pR_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_pR_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_pR_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_pR_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_conj_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_conj_P");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_conj_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_conj_pP");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_i_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_i_P");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_i_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_i_pP");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_Pa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_pPa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_transpose_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_transpose_P");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_transpose_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_transpose_pP");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_P");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_pP");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_veqm_c_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_c_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_r_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_r_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_c_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_c_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_r_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_r_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_c_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_c_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_r_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_r_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_c_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_c_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_r_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_r_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_C_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_C_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_C_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_C_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_C_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_C_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_C_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_C_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_pC_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_pC_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_pC_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_pC_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_pC_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_pC_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_pC_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_pC_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_Ca_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_Ca_times_P");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_Ca_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_Ca_times_pP");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_Ca_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_Ca_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_Ca_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_Ca_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_pCa_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_pCa_times_P");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_pCa_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_pCa_times_pP");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_pCa_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_pCa_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_pCa_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_pCa_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_R_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_R_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_R_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_R_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_R_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_R_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_R_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_R_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_pR_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_pR_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_pR_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_pR_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_pR_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_pR_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_pR_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_pR_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_conj_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_conj_P");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_conj_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_conj_pP");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_i_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_i_P");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_i_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_i_pP");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_Pa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_pPa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_transpose_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_transpose_P");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_transpose_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_transpose_pP");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_P");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veqm_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_pP");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veq_P_plus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_P_plus_P");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_r_times_P_plus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, QLA_F2_DiracPropagator *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F2_P_veq_r_times_P_plus_P");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_c_times_P_plus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, QLA_F2_DiracPropagator *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F2_P_veq_c_times_P_plus_P");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_P_minus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_P_minus_P");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_r_times_P_minus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, QLA_F2_DiracPropagator *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F2_P_veq_r_times_P_minus_P");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_c_times_P_minus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, QLA_F2_DiracPropagator *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F2_P_veq_c_times_P_minus_P");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_P_plus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_P_plus_pP");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_r_times_P_plus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, QLA_F2_DiracPropagator *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F2_P_veq_r_times_P_plus_pP");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_c_times_P_plus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, QLA_F2_DiracPropagator *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F2_P_veq_c_times_P_plus_pP");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_P_minus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_P_minus_pP");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_r_times_P_minus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, QLA_F2_DiracPropagator *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F2_P_veq_r_times_P_minus_pP");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_c_times_P_minus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, QLA_F2_DiracPropagator *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F2_P_veq_c_times_P_minus_pP");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pP_plus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pP_plus_P");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_r_times_pP_plus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, QLA_F2_DiracPropagator *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F2_P_veq_r_times_pP_plus_P");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_c_times_pP_plus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, QLA_F2_DiracPropagator *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F2_P_veq_c_times_pP_plus_P");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pP_minus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pP_minus_P");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_r_times_pP_minus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, QLA_F2_DiracPropagator *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F2_P_veq_r_times_pP_minus_P");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_c_times_pP_minus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, QLA_F2_DiracPropagator *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F2_P_veq_c_times_pP_minus_P");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pP_plus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pP_plus_pP");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_r_times_pP_plus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, QLA_F2_DiracPropagator *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F2_P_veq_r_times_pP_plus_pP");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_c_times_pP_plus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, QLA_F2_DiracPropagator *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F2_P_veq_c_times_pP_plus_pP");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_pP_minus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pP_minus_pP");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_r_times_pP_minus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, QLA_F2_DiracPropagator *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F2_P_veq_r_times_pP_minus_pP");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_veq_c_times_pP_minus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, QLA_F2_DiracPropagator *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F2_P_veq_c_times_pP_minus_pP");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_c_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_c_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_r_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_r_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_c_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_c_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_r_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_r_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_c_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_c_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_r_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_r_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_c_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_c_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_r_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_r_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_C_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_C_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_C_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_C_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_C_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_C_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_C_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_C_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pC_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pC_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pC_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pC_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pC_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pC_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pC_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pC_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_Ca_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_Ca_times_P");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_Ca_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_Ca_times_pP");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_Ca_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_Ca_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_Ca_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_Ca_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pCa_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pCa_times_P");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pCa_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pCa_times_pP");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pCa_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pCa_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pCa_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pCa_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_R_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_R_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_R_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_R_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_R_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_R_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_R_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_R_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pR_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pR_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pR_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pR_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pR_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pR_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pR_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pR_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_conj_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_conj_P");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_conj_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_conj_pP");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_i_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_i_P");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_i_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_i_pP");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_Pa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pPa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_transpose_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_transpose_P");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_transpose_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_transpose_pP");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_P");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pP");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_c_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_c_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_r_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_r_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_c_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_c_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_r_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_r_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_c_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_c_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_r_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_r_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_c_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_c_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_r_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_r_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_C_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_C_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_C_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_C_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_C_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_C_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_C_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_C_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_pC_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_pC_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_pC_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_pC_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_pC_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_pC_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_pC_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_pC_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_Ca_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_Ca_times_P");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_Ca_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_Ca_times_pP");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_Ca_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_Ca_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_Ca_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_Ca_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_pCa_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_pCa_times_P");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_pCa_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_pCa_times_pP");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_pCa_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_pCa_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_pCa_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_pCa_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_R_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_R_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_R_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_R_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_R_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_R_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_R_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_R_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_pR_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_pR_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_pR_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_pR_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_pR_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_pR_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_pR_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_pR_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_conj_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_conj_P");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_conj_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_conj_pP");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_i_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_i_P");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_i_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_i_pP");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_Pa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_pPa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_transpose_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_transpose_P");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_transpose_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_transpose_pP");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_P");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_pP");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_c_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_c_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_r_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_r_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_c_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_c_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_r_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_r_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_c_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_c_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_r_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_r_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_c_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_c_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_r_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_r_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_C_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_C_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_C_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_C_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_C_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_C_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_C_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_C_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_pC_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_pC_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_pC_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_pC_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_pC_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_pC_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_pC_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_pC_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_Ca_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_Ca_times_P");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_Ca_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_Ca_times_pP");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_Ca_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_Ca_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_Ca_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_Ca_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_pCa_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_pCa_times_P");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_pCa_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_pCa_times_pP");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_pCa_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_pCa_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_pCa_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_pCa_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_R_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_R_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_R_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_R_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_R_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_R_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_R_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_R_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_pR_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_pR_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_pR_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_pR_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_pR_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_pR_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_pR_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_pR_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_conj_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_conj_P");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_conj_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_conj_pP");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_i_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_i_P");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_i_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_i_pP");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_Pa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_pPa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_transpose_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_transpose_P");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_transpose_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_transpose_pP");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_P");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_pP");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xeqm_c_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_c_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_r_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_r_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_c_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_c_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_r_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_r_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_c_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_c_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_r_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_r_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_c_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_c_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_r_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_r_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("F2_ew_rtimes", 2, 16 * 2 * 2, qlab::PERM_P, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_C_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_C_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_C_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_C_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_C_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_C_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_C_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_C_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_pC_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_pC_times_P");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_pC_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_pC_times_pP");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_pC_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_pC_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_pC_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_pC_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_Ca_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_Ca_times_P");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_Ca_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_Ca_times_pP");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_Ca_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_Ca_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_Ca_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_Ca_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_pCa_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_pCa_times_P");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_pCa_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_pCa_times_pP");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_pCa_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_pCa_times_Pa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_pCa_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_pCa_times_pPa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_R_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_R_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_R_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_R_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_R_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_R_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_R_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_R_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_pR_times_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_pR_times_P");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_pR_times_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_pR_times_pP");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_pR_times_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_pR_times_Pa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_pR_times_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_pR_times_pPa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("F2_ew_field", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_conj_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_conj_P");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_conj_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_conj_pP");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_i_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_i_P");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_i_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_i_pP");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_Pa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_Pa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_pPa(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_pPa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_transpose_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_transpose_P");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_transpose_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_transpose_pP");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_P, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_P");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeqm_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_pP");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("F2_ew_unary", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeq_P_plus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_P_plus_P");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_r_times_P_plus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, QLA_F2_DiracPropagator *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_r_times_P_plus_P");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_c_times_P_plus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, QLA_F2_DiracPropagator *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_c_times_P_plus_P");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_P_minus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_P_minus_P");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_r_times_P_minus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, QLA_F2_DiracPropagator *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_r_times_P_minus_P");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_c_times_P_minus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, QLA_F2_DiracPropagator *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_c_times_P_minus_P");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_P_plus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_P_plus_pP");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_r_times_P_plus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, QLA_F2_DiracPropagator *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_r_times_P_plus_pP");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_c_times_P_plus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, QLA_F2_DiracPropagator *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_c_times_P_plus_pP");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_P_minus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_P_minus_pP");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_r_times_P_minus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, QLA_F2_DiracPropagator *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_r_times_P_minus_pP");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_c_times_P_minus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, QLA_F2_DiracPropagator *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_c_times_P_minus_pP");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pP_plus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pP_plus_P");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_r_times_pP_plus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, QLA_F2_DiracPropagator *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_r_times_pP_plus_P");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_c_times_pP_plus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, QLA_F2_DiracPropagator *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_c_times_pP_plus_P");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pP_minus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pP_minus_P");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_r_times_pP_minus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, QLA_F2_DiracPropagator *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_r_times_pP_minus_P");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_c_times_pP_minus_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, QLA_F2_DiracPropagator *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_c_times_pP_minus_P");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pP_plus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pP_plus_pP");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_r_times_pP_plus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, QLA_F2_DiracPropagator *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_r_times_pP_plus_pP");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_c_times_pP_plus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, QLA_F2_DiracPropagator *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_c_times_pP_plus_pP");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_pP_minus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pP_minus_pP");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 16 * 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_r_times_pP_minus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, QLA_F2_DiracPropagator *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_r_times_pP_minus_pP");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xeq_c_times_pP_minus_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, QLA_F2_DiracPropagator *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_c_times_pP_minus_pP");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 16 * 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

}  // extern "C"
