// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F2 ewise_v entry points (extern "C"), reference: lib/perl/build_qla.pl:403-469, 1256-1420 (element-wise families)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_F2_V_veq_c_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_c_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_c_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_c_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_C_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_C_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_C_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_C_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_pC_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_pC_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_pC_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_pC_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_Ca_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_Ca_times_V");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_Ca_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_Ca_times_pV");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_pCa_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_pCa_times_V");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_pCa_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_pCa_times_pV");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_R_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_R_times_V");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_R_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_R_times_pV");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_pR_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_pR_times_V");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_pR_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_pR_times_pV");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_conj_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_V_veq_conj_V");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_conj_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_V_veq_conj_pV");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_i_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_V_veq_i_V");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_i_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_V_veq_i_pV");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_c_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_c_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_c_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_c_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_C_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_C_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_C_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_C_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_pC_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_pC_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_pC_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_pC_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_Ca_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_Ca_times_V");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_Ca_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_Ca_times_pV");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_pCa_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_pCa_times_V");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_pCa_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_pCa_times_pV");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_R_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_R_times_V");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_R_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_R_times_pV");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_pR_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_pR_times_V");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_pR_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_pR_times_pV");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_conj_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_conj_V");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_conj_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_conj_pV");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_i_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_i_V");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_i_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_i_pV");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_c_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_c_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_c_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_c_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_C_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_C_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_C_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_C_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_pC_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_pC_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_pC_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_pC_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_Ca_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_Ca_times_V");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_Ca_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_Ca_times_pV");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_pCa_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_pCa_times_V");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_pCa_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_pCa_times_pV");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_R_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_R_times_V");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_R_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_R_times_pV");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_pR_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_pR_times_V");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_pR_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_pR_times_pV");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_conj_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_conj_V");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_conj_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_conj_pV");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_i_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_i_V");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_i_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_i_pV");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_veqm_c_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_c_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_c_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_c_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_C_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_C_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_C_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_C_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_pC_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_pC_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_pC_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_pC_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_Ca_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_Ca_times_V");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_Ca_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_Ca_times_pV");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_pCa_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_pCa_times_V");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_pCa_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_pCa_times_pV");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_R_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_R_times_V");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_R_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_R_times_pV");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_pR_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_pR_times_V");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_pR_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_pR_times_pV");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_conj_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_conj_V");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_conj_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_conj_pV");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_i_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_i_V");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_i_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_i_pV");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veq_V_plus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_V_plus_V");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_r_times_V_plus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, QLA_F2_ColorVector *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_r_times_V_plus_V");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_c_times_V_plus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, QLA_F2_ColorVector *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_c_times_V_plus_V");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_V_minus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_V_minus_V");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_r_times_V_minus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, QLA_F2_ColorVector *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_r_times_V_minus_V");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_c_times_V_minus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, QLA_F2_ColorVector *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_c_times_V_minus_V");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_V_plus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_V_plus_pV");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_r_times_V_plus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, QLA_F2_ColorVector *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_r_times_V_plus_pV");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_c_times_V_plus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, QLA_F2_ColorVector *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_c_times_V_plus_pV");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_V_minus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_V_minus_pV");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_r_times_V_minus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, QLA_F2_ColorVector *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_r_times_V_minus_pV");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_c_times_V_minus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, QLA_F2_ColorVector *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_c_times_V_minus_pV");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_pV_plus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_pV_plus_V");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_r_times_pV_plus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, QLA_F2_ColorVector *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_r_times_pV_plus_V");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_c_times_pV_plus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, QLA_F2_ColorVector *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_c_times_pV_plus_V");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_pV_minus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_pV_minus_V");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_r_times_pV_minus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, QLA_F2_ColorVector *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_r_times_pV_minus_V");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_c_times_pV_minus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, QLA_F2_ColorVector *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_c_times_pV_minus_V");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_pV_plus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_pV_plus_pV");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_r_times_pV_plus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, QLA_F2_ColorVector *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_r_times_pV_plus_pV");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_c_times_pV_plus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, QLA_F2_ColorVector *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_c_times_pV_plus_pV");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_pV_minus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_pV_minus_pV");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_r_times_pV_minus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, QLA_F2_ColorVector *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_r_times_pV_minus_pV");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_c_times_pV_minus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, QLA_F2_ColorVector *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_c_times_pV_minus_pV");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_c_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_c_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_c_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_c_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_C_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_C_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_C_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_C_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_pC_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_pC_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_pC_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_pC_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_Ca_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_Ca_times_V");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_Ca_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_Ca_times_pV");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_pCa_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_pCa_times_V");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_pCa_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_pCa_times_pV");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_R_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_R_times_V");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_R_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_R_times_pV");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_pR_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_pR_times_V");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_pR_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_pR_times_pV");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_conj_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_conj_V");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_conj_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_conj_pV");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_i_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_i_V");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_i_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_i_pV");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_c_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_c_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_c_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_c_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_C_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_C_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_C_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_C_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_pC_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_pC_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_pC_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_pC_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_Ca_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_Ca_times_V");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_Ca_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_Ca_times_pV");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_pCa_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_pCa_times_V");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_pCa_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_pCa_times_pV");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_R_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_R_times_V");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_R_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_R_times_pV");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_pR_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_pR_times_V");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_pR_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_pR_times_pV");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_conj_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_conj_V");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_conj_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_conj_pV");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_i_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_i_V");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_i_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_i_pV");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_c_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_c_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_c_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_c_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_C_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_C_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_C_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_C_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_pC_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_pC_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_pC_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_pC_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_Ca_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_Ca_times_V");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_Ca_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_Ca_times_pV");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_pCa_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_pCa_times_V");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_pCa_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_pCa_times_pV");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_R_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_R_times_V");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_R_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_R_times_pV");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_pR_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_pR_times_V");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_pR_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_pR_times_pV");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_conj_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_conj_V");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_conj_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_conj_pV");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_i_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_i_V");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_i_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_i_pV");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xeqm_c_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_c_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_c_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_c_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("F2_ew_ctimes", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_C_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_C_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_C_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_C_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_pC_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_pC_times_V");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_pC_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_pC_times_pV");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_Ca_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_Ca_times_V");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_Ca_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_Ca_times_pV");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_pCa_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_pCa_times_V");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_pCa_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_pCa_times_pV");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_R_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_R_times_V");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_R_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_R_times_pV");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_pR_times_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_pR_times_V");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_pR_times_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_pR_times_pV");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("F2_ew_field", 2, 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_conj_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_conj_V");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_conj_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_conj_pV");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_i_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_i_V");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_i_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_i_pV");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("F2_ew_unary", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeq_V_plus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_V_plus_V");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_r_times_V_plus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, QLA_F2_ColorVector *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_r_times_V_plus_V");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_c_times_V_plus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, QLA_F2_ColorVector *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_c_times_V_plus_V");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_V_minus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_V_minus_V");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_r_times_V_minus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, QLA_F2_ColorVector *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_r_times_V_minus_V");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_c_times_V_minus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, QLA_F2_ColorVector *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_c_times_V_minus_V");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_V_plus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_V_plus_pV");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_r_times_V_plus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, QLA_F2_ColorVector *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_r_times_V_plus_pV");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_c_times_V_plus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, QLA_F2_ColorVector *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_c_times_V_plus_pV");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_V_minus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_V_minus_pV");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_r_times_V_minus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, QLA_F2_ColorVector *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_r_times_V_minus_pV");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_c_times_V_minus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, QLA_F2_ColorVector *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_c_times_V_minus_pV");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_pV_plus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_pV_plus_V");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_r_times_pV_plus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, QLA_F2_ColorVector *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_r_times_pV_plus_V");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_c_times_pV_plus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, QLA_F2_ColorVector *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_c_times_pV_plus_V");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_pV_minus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_pV_minus_V");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_r_times_pV_minus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, QLA_F2_ColorVector *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_r_times_pV_minus_V");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_c_times_pV_minus_V(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, QLA_F2_ColorVector *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_c_times_pV_minus_V");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_pV_plus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_pV_plus_pV");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_r_times_pV_plus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, QLA_F2_ColorVector *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_r_times_pV_plus_pV");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_c_times_pV_plus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, QLA_F2_ColorVector *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_c_times_pV_plus_pV");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_pV_minus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_pV_minus_pV");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("F2_ew_sum", 2, 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_r_times_pV_minus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, QLA_F2_ColorVector *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_r_times_pV_minus_pV");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_c_times_pV_minus_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, QLA_F2_ColorVector *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_c_times_pV_minus_pV");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("F2_ew_axpby", 2, 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

}  // extern "C"
