// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA FN ewise_m entry points (extern "C"), reference: lib/perl/build_qla.pl:403-469, 1256-1420 (element-wise families)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_FN_M_veq_c_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_c_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_c_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_c_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_c_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_c_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_r_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_r_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("FN_ew_rtimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_c_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_c_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_r_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_r_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("FN_ew_rtimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_C_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_C_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_C_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_C_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_C_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_C_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_C_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_C_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pC_times_M(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pC_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pC_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pC_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pC_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pC_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pC_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pC_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_Ca_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_Ca_times_M");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_Ca_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_Ca_times_pM");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_Ca_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_Ca_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_Ca_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_Ca_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pCa_times_M(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pCa_times_M");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pCa_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pCa_times_pM");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pCa_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pCa_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pCa_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pCa_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_R_times_M(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_R_times_M");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_R_times_pM(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_R_times_pM");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_R_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_R_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_R_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_R_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pR_times_M(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pR_times_M");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pR_times_pM(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pR_times_pM");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pR_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pR_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pR_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pR_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_conj_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_conj_M");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_conj_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_conj_pM");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_i_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_i_M");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_i_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_i_pM");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_Ma(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_Ma");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pMa(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pMa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_transpose_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_transpose_M");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_transpose_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_transpose_pM");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_c_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_c_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_c_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_c_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_c_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_c_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_r_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_r_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("FN_ew_rtimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_c_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_c_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_r_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_r_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("FN_ew_rtimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_C_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_C_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_C_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_C_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_C_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_C_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_C_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_C_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_pC_times_M(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pC_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_pC_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pC_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_pC_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pC_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_pC_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pC_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_Ca_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_Ca_times_M");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_Ca_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_Ca_times_pM");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_Ca_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_Ca_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_Ca_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_Ca_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_pCa_times_M(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pCa_times_M");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_pCa_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pCa_times_pM");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_pCa_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pCa_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_pCa_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pCa_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_R_times_M(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_R_times_M");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_R_times_pM(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_R_times_pM");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_R_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_R_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_R_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_R_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_pR_times_M(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pR_times_M");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_pR_times_pM(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pR_times_pM");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_pR_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pR_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_pR_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pR_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_conj_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_conj_M");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_conj_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_conj_pM");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_i_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_i_M");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_i_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_i_pM");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_Ma(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_Ma");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_pMa(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pMa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_transpose_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_transpose_M");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vpeq_transpose_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_transpose_pM");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_c_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_c_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_c_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_c_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_c_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_c_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_r_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_r_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("FN_ew_rtimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_c_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_c_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_r_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_r_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("FN_ew_rtimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_C_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_C_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_C_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_C_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_C_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_C_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_C_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_C_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_pC_times_M(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pC_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_pC_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pC_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_pC_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pC_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_pC_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pC_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_Ca_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_Ca_times_M");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_Ca_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_Ca_times_pM");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_Ca_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_Ca_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_Ca_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_Ca_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_pCa_times_M(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pCa_times_M");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_pCa_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pCa_times_pM");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_pCa_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pCa_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_pCa_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pCa_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_R_times_M(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_R_times_M");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_R_times_pM(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_R_times_pM");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_R_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_R_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_R_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_R_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_pR_times_M(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pR_times_M");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_pR_times_pM(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pR_times_pM");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_pR_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pR_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_pR_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pR_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_conj_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_conj_M");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_conj_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_conj_pM");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_i_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_i_M");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_i_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_i_pM");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_Ma(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_Ma");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_pMa(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pMa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_transpose_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_transpose_M");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_vmeq_transpose_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_transpose_pM");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_veqm_c_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_c_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_c_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_c_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_c_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_c_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_r_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_r_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("FN_ew_rtimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_c_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_c_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_r_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_r_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("FN_ew_rtimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_C_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_C_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_C_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_C_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_C_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_C_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_C_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_C_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_pC_times_M(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pC_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_pC_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pC_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_pC_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pC_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_pC_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pC_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_Ca_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_Ca_times_M");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_Ca_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_Ca_times_pM");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_Ca_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_Ca_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_Ca_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_Ca_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_pCa_times_M(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pCa_times_M");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_pCa_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pCa_times_pM");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_pCa_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pCa_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_pCa_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pCa_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_R_times_M(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_R_times_M");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_R_times_pM(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_R_times_pM");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_R_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_R_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_R_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_R_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_pR_times_M(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pR_times_M");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_pR_times_pM(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pR_times_pM");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_pR_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pR_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_pR_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pR_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_conj_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_conj_M");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_conj_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_conj_pM");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_i_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_i_M");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_i_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_i_pM");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_Ma(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_Ma");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_pMa(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pMa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_transpose_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_transpose_M");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veqm_transpose_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_transpose_pM");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_veq_M_plus_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_M_plus_M");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("FN_ew_sum", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_r_times_M_plus_M(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, void * c, int n) {
  QLAB_TRACE("QLA_FN_M_veq_r_times_M_plus_M");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_c_times_M_plus_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, void * c, int n) {
  QLAB_TRACE("QLA_FN_M_veq_c_times_M_plus_M");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_M_minus_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_M_minus_M");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("FN_ew_sum", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_r_times_M_minus_M(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, void * c, int n) {
  QLAB_TRACE("QLA_FN_M_veq_r_times_M_minus_M");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_c_times_M_minus_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, void * c, int n) {
  QLAB_TRACE("QLA_FN_M_veq_c_times_M_minus_M");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_M_plus_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_M_plus_pM");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("FN_ew_sum", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_r_times_M_plus_pM(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, void * c, int n) {
  QLAB_TRACE("QLA_FN_M_veq_r_times_M_plus_pM");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_c_times_M_plus_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, void * c, int n) {
  QLAB_TRACE("QLA_FN_M_veq_c_times_M_plus_pM");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_M_minus_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_M_minus_pM");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("FN_ew_sum", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_r_times_M_minus_pM(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, void * c, int n) {
  QLAB_TRACE("QLA_FN_M_veq_r_times_M_minus_pM");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_c_times_M_minus_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, void * c, int n) {
  QLAB_TRACE("QLA_FN_M_veq_c_times_M_minus_pM");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pM_plus_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pM_plus_M");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("FN_ew_sum", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_r_times_pM_plus_M(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, void * c, int n) {
  QLAB_TRACE("QLA_FN_M_veq_r_times_pM_plus_M");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_c_times_pM_plus_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, void * c, int n) {
  QLAB_TRACE("QLA_FN_M_veq_c_times_pM_plus_M");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pM_minus_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pM_minus_M");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("FN_ew_sum", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_r_times_pM_minus_M(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, void * c, int n) {
  QLAB_TRACE("QLA_FN_M_veq_r_times_pM_minus_M");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_c_times_pM_minus_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, void * c, int n) {
  QLAB_TRACE("QLA_FN_M_veq_c_times_pM_minus_M");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pM_plus_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pM_plus_pM");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("FN_ew_sum", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_r_times_pM_plus_pM(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, void * c, int n) {
  QLAB_TRACE("QLA_FN_M_veq_r_times_pM_plus_pM");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_c_times_pM_plus_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, void * c, int n) {
  QLAB_TRACE("QLA_FN_M_veq_c_times_pM_plus_pM");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_pM_minus_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pM_minus_pM");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("FN_ew_sum", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_r_times_pM_minus_pM(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, void * c, int n) {
  QLAB_TRACE("QLA_FN_M_veq_r_times_pM_minus_pM");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_veq_c_times_pM_minus_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, void * c, int n) {
  QLAB_TRACE("QLA_FN_M_veq_c_times_pM_minus_pM");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_c_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_c_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_c_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_c_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_c_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_c_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_r_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_r_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("FN_ew_rtimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_c_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_c_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_r_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_r_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("FN_ew_rtimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_C_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_C_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_C_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_C_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_C_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_C_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_C_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_C_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pC_times_M(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pC_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pC_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pC_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pC_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pC_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pC_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pC_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_Ca_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_Ca_times_M");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_Ca_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_Ca_times_pM");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_Ca_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_Ca_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_Ca_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_Ca_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pCa_times_M(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pCa_times_M");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pCa_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pCa_times_pM");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pCa_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pCa_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pCa_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pCa_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_R_times_M(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_R_times_M");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_R_times_pM(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_R_times_pM");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_R_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_R_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_R_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_R_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pR_times_M(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pR_times_M");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pR_times_pM(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pR_times_pM");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pR_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pR_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pR_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pR_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_conj_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_conj_M");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_conj_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_conj_pM");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_i_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_i_M");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_i_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_i_pM");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_Ma(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_Ma");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pMa(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pMa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_transpose_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_transpose_M");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_transpose_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_transpose_pM");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_c_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_c_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_c_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_c_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_c_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_c_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_r_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_r_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("FN_ew_rtimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_c_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_c_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_r_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_r_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("FN_ew_rtimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_C_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_C_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_C_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_C_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_C_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_C_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_C_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_C_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_pC_times_M(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pC_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_pC_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pC_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_pC_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pC_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_pC_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pC_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_Ca_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_Ca_times_M");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_Ca_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_Ca_times_pM");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_Ca_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_Ca_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_Ca_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_Ca_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_pCa_times_M(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pCa_times_M");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_pCa_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pCa_times_pM");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_pCa_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pCa_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_pCa_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pCa_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_R_times_M(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_R_times_M");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_R_times_pM(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_R_times_pM");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_R_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_R_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_R_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_R_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_pR_times_M(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pR_times_M");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_pR_times_pM(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pR_times_pM");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_pR_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pR_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_pR_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pR_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_conj_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_conj_M");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_conj_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_conj_pM");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_i_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_i_M");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_i_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_i_pM");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_Ma(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_Ma");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_pMa(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pMa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_transpose_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_transpose_M");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xpeq_transpose_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_transpose_pM");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_c_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_c_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_c_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_c_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_c_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_c_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_r_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_r_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("FN_ew_rtimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_c_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_c_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_r_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_r_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("FN_ew_rtimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_C_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_C_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_C_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_C_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_C_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_C_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_C_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_C_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_pC_times_M(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pC_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_pC_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pC_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_pC_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pC_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_pC_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pC_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_Ca_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_Ca_times_M");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_Ca_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_Ca_times_pM");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_Ca_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_Ca_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_Ca_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_Ca_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_pCa_times_M(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pCa_times_M");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_pCa_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pCa_times_pM");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_pCa_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pCa_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_pCa_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pCa_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_R_times_M(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_R_times_M");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_R_times_pM(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_R_times_pM");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_R_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_R_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_R_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_R_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_pR_times_M(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pR_times_M");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_pR_times_pM(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pR_times_pM");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_pR_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pR_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_pR_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pR_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_conj_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_conj_M");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_conj_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_conj_pM");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_i_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_i_M");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_i_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_i_pM");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_Ma(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_Ma");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_pMa(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pMa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_transpose_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_transpose_M");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xmeq_transpose_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_transpose_pM");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_FN_M_xeqm_c_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_c_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_c_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_c_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_c_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_c_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_r_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_r_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("FN_ew_rtimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_c_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_c_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_CONST, false>("FN_ew_ctimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_r_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_r_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_CONST, true>("FN_ew_rtimes", nc, nc * nc, qlab::PERM_M, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_C_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_C_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_C_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_C_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_C_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_C_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_C_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_C_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_pC_times_M(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pC_times_M");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_pC_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pC_times_pM");
  qlab::api_ew_n<float, qlab::EW_CT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_pC_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pC_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_pC_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pC_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CTA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_Ca_times_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_Ca_times_M");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_Ca_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_Ca_times_pM");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_Ca_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_Ca_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_Ca_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_Ca_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_pCa_times_M(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pCa_times_M");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_pCa_times_pM(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pCa_times_pM");
  qlab::api_ew_n<float, qlab::EW_CAT, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_pCa_times_Ma(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pCa_times_Ma");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_pCa_times_pMa(int nc, void * r, QLA_F_Complex *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pCa_times_pMa");
  qlab::api_ew_n<float, qlab::EW_CATA, qlab::SC_FIELD, false>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_R_times_M(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_R_times_M");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_R_times_pM(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_R_times_pM");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_R_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_R_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_R_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_R_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_pR_times_M(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pR_times_M");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_pR_times_pM(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pR_times_pM");
  qlab::api_ew_n<float, qlab::EW_RT, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_pR_times_Ma(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pR_times_Ma");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_pR_times_pMa(int nc, void * r, QLA_F_Real *__restrict__ * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pR_times_pMa");
  qlab::api_ew_n<float, qlab::EW_RTA, qlab::SC_FIELD, true>("FN_ew_field", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_conj_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_conj_M");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_conj_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_conj_pM");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_i_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_i_M");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_i_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_i_pM");
  qlab::api_ew_n<float, qlab::EW_I, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_Ma(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_Ma");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_pMa(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pMa");
  qlab::api_ew_n<float, qlab::EW_CONJ, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_transpose_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_transpose_M");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeqm_transpose_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_transpose_pM");
  qlab::api_ew_n<float, qlab::EW_COPY, qlab::SC_NONE, false>("FN_ew_unary", nc, nc * nc, qlab::PERM_M, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_FN_M_xeq_M_plus_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_M_plus_M");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("FN_ew_sum", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_r_times_M_plus_M(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, void * c, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_r_times_M_plus_M");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_c_times_M_plus_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, void * c, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_c_times_M_plus_M");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_M_minus_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_M_minus_M");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("FN_ew_sum", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_r_times_M_minus_M(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, void * c, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_r_times_M_minus_M");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_c_times_M_minus_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, void * c, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_c_times_M_minus_M");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_M_plus_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_M_plus_pM");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("FN_ew_sum", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_r_times_M_plus_pM(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, void * c, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_r_times_M_plus_pM");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_c_times_M_plus_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, void * c, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_c_times_M_plus_pM");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_M_minus_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_M_minus_pM");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("FN_ew_sum", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_r_times_M_minus_pM(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, void * c, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_r_times_M_minus_pM");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_c_times_M_minus_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, void * c, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_c_times_M_minus_pM");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pM_plus_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pM_plus_M");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("FN_ew_sum", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_r_times_pM_plus_M(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, void * c, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_r_times_pM_plus_M");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_c_times_pM_plus_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, void * c, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_c_times_pM_plus_M");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pM_minus_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pM_minus_M");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("FN_ew_sum", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_r_times_pM_minus_M(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, void * c, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_r_times_pM_minus_M");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_c_times_pM_minus_M(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, void * c, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_c_times_pM_minus_M");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pM_plus_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pM_plus_pM");
  qlab::api_ew_n<float, qlab::EW_PLUS, qlab::SC_NONE, false>("FN_ew_sum", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_r_times_pM_plus_pM(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, void * c, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_r_times_pM_plus_pM");
  qlab::api_ew_n<float, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_c_times_pM_plus_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, void * c, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_c_times_pM_plus_pM");
  qlab::api_ew_n<float, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_pM_minus_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pM_minus_pM");
  qlab::api_ew_n<float, qlab::EW_MINUS, qlab::SC_NONE, false>("FN_ew_sum", nc, nc * nc, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_r_times_pM_minus_pM(int nc, void * r, QLA_F_Real *__restrict__ a, void * b, void * c, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_r_times_pM_minus_pM");
  qlab::api_ew_n<float, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_FN_M_xeq_c_times_pM_minus_pM(int nc, void * r, QLA_F_Complex *__restrict__ a, void * b, void * c, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_c_times_pM_minus_pM");
  qlab::api_ew_n<float, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("FN_ew_axpby", nc, nc * nc, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

}  // extern "C"
