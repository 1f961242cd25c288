// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F sglobal entry points (extern "C"), reference: lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_scalar.cuh"

extern "C" {
QLAB_EXPORT void QLA_F_c_veq_C_dot_C(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_c_veq_C_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_DOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F_c_veq_C_dot_pC(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_c_veq_C_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_DOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F_c_veq_pC_dot_C(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_c_veq_pC_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_DOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F_c_veq_pC_dot_pC(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_c_veq_pC_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_DOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F_c_xeq_C_dot_C(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_c_xeq_C_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_DOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F_c_xeq_C_dot_pC(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_c_xeq_C_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_DOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F_c_xeq_pC_dot_C(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_c_xeq_pC_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_DOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F_c_xeq_pC_dot_pC(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_c_xeq_pC_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_DOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F_c_veq_Ca_dot_C(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_c_veq_Ca_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_ADOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F_c_veq_Ca_dot_pC(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_c_veq_Ca_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_ADOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F_c_veq_pCa_dot_C(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_c_veq_pCa_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_ADOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F_c_veq_pCa_dot_pC(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_c_veq_pCa_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_ADOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F_c_xeq_Ca_dot_C(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_c_xeq_Ca_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_ADOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F_c_xeq_Ca_dot_pC(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_c_xeq_Ca_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_ADOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F_c_xeq_pCa_dot_C(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_c_xeq_pCa_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_ADOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F_c_xeq_pCa_dot_pC(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_c_xeq_pCa_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_ADOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F_c_veq_sum_C(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_c_veq_sum_C");
  qlab::api_gsum<float, 1, float>("F_gsum", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_F_c_veq_sum_pC(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_c_veq_sum_pC");
  qlab::api_gsum<float, 1, float>("F_gsum", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_F_c_xeq_sum_C(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_c_xeq_sum_C");
  qlab::api_gsum<float, 1, float>("F_gsum", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_F_c_xeq_sum_pC(QLA_F_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_c_xeq_sum_pC");
  qlab::api_gsum<float, 1, float>("F_gsum", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_F_r_veq_R_dot_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_r_veq_R_dot_R");
  qlab::api_sred<float, float, qlab::SR_DOT, float>("F_sred", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F_r_veq_R_dot_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_r_veq_R_dot_pR");
  qlab::api_sred<float, float, qlab::SR_DOT, float>("F_sred", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F_r_veq_pR_dot_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_r_veq_pR_dot_R");
  qlab::api_sred<float, float, qlab::SR_DOT, float>("F_sred", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F_r_veq_pR_dot_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_r_veq_pR_dot_pR");
  qlab::api_sred<float, float, qlab::SR_DOT, float>("F_sred", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F_r_xeq_R_dot_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_R_dot_R");
  qlab::api_sred<float, float, qlab::SR_DOT, float>("F_sred", r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F_r_xeq_R_dot_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_R_dot_pR");
  qlab::api_sred<float, float, qlab::SR_DOT, float>("F_sred", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F_r_xeq_pR_dot_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_pR_dot_R");
  qlab::api_sred<float, float, qlab::SR_DOT, float>("F_sred", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F_r_xeq_pR_dot_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_pR_dot_pR");
  qlab::api_sred<float, float, qlab::SR_DOT, float>("F_sred", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F_r_veq_I_dot_I(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_r_veq_I_dot_I");
  qlab::api_sred<int, float, qlab::SR_DOT, float>("F_sred", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F_r_veq_I_dot_pI(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_r_veq_I_dot_pI");
  qlab::api_sred<int, float, qlab::SR_DOT, float>("F_sred", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F_r_veq_pI_dot_I(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_r_veq_pI_dot_I");
  qlab::api_sred<int, float, qlab::SR_DOT, float>("F_sred", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F_r_veq_pI_dot_pI(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_r_veq_pI_dot_pI");
  qlab::api_sred<int, float, qlab::SR_DOT, float>("F_sred", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F_r_xeq_I_dot_I(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_I_dot_I");
  qlab::api_sred<int, float, qlab::SR_DOT, float>("F_sred", r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F_r_xeq_I_dot_pI(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_I_dot_pI");
  qlab::api_sred<int, float, qlab::SR_DOT, float>("F_sred", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F_r_xeq_pI_dot_I(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_pI_dot_I");
  qlab::api_sred<int, float, qlab::SR_DOT, float>("F_sred", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F_r_xeq_pI_dot_pI(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_pI_dot_pI");
  qlab::api_sred<int, float, qlab::SR_DOT, float>("F_sred", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F_r_veq_norm2_C(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_r_veq_norm2_C");
  qlab::api_gdot<float, 1, qlab::LD_NORM2, qlab::PERM_ID, float>("F_gdot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F_r_veq_norm2_pC(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_r_veq_norm2_pC");
  qlab::api_gdot<float, 1, qlab::LD_NORM2, qlab::PERM_ID, float>("F_gdot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F_r_xeq_norm2_C(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_norm2_C");
  qlab::api_gdot<float, 1, qlab::LD_NORM2, qlab::PERM_ID, float>("F_gdot", r, qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F_r_xeq_norm2_pC(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_norm2_pC");
  qlab::api_gdot<float, 1, qlab::LD_NORM2, qlab::PERM_ID, float>("F_gdot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F_r_veq_norm2_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_r_veq_norm2_R");
  qlab::api_sred<float, float, qlab::SR_NORM2, float>("F_sred", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F_r_veq_norm2_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_r_veq_norm2_pR");
  qlab::api_sred<float, float, qlab::SR_NORM2, float>("F_sred", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F_r_xeq_norm2_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_norm2_R");
  qlab::api_sred<float, float, qlab::SR_NORM2, float>("F_sred", r, qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F_r_xeq_norm2_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_norm2_pR");
  qlab::api_sred<float, float, qlab::SR_NORM2, float>("F_sred", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F_r_veq_norm2_I(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_r_veq_norm2_I");
  qlab::api_sred<int, float, qlab::SR_NORM2, float>("F_sred", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F_r_veq_norm2_pI(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_r_veq_norm2_pI");
  qlab::api_sred<int, float, qlab::SR_NORM2, float>("F_sred", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F_r_xeq_norm2_I(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_norm2_I");
  qlab::api_sred<int, float, qlab::SR_NORM2, float>("F_sred", r, qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F_r_xeq_norm2_pI(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_norm2_pI");
  qlab::api_sred<int, float, qlab::SR_NORM2, float>("F_sred", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F_r_veq_re_C_dot_C(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_r_veq_re_C_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_REDOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F_r_veq_re_C_dot_pC(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_r_veq_re_C_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_REDOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F_r_veq_re_pC_dot_C(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_r_veq_re_pC_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_REDOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F_r_veq_re_pC_dot_pC(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_r_veq_re_pC_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_REDOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F_r_xeq_re_C_dot_C(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_re_C_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_REDOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F_r_xeq_re_C_dot_pC(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_re_C_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_REDOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F_r_xeq_re_pC_dot_C(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_re_pC_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_REDOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F_r_xeq_re_pC_dot_pC(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_re_pC_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_REDOT, qlab::PERM_ID, float>("F_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F_r_veq_sum_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_r_veq_sum_R");
  qlab::api_sred<float, float, qlab::SR_SUM, float>("F_sred", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F_r_veq_sum_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_r_veq_sum_pR");
  qlab::api_sred<float, float, qlab::SR_SUM, float>("F_sred", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F_r_xeq_sum_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_sum_R");
  qlab::api_sred<float, float, qlab::SR_SUM, float>("F_sred", r, qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F_r_xeq_sum_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_sum_pR");
  qlab::api_sred<float, float, qlab::SR_SUM, float>("F_sred", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F_r_veq_sum_I(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_r_veq_sum_I");
  qlab::api_sred<int, float, qlab::SR_SUM, float>("F_sred", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F_r_veq_sum_pI(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_r_veq_sum_pI");
  qlab::api_sred<int, float, qlab::SR_SUM, float>("F_sred", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F_r_xeq_sum_I(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_sum_I");
  qlab::api_sred<int, float, qlab::SR_SUM, float>("F_sred", r, qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F_r_xeq_sum_pI(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_r_xeq_sum_pI");
  qlab::api_sred<int, float, qlab::SR_SUM, float>("F_sred", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DF_c_veq_C_dot_C(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF_c_veq_C_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_DOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF_c_veq_C_dot_pC(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF_c_veq_C_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_DOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF_c_veq_pC_dot_C(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF_c_veq_pC_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_DOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF_c_veq_pC_dot_pC(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF_c_veq_pC_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_DOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF_c_xeq_C_dot_C(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF_c_xeq_C_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_DOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF_c_xeq_C_dot_pC(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF_c_xeq_C_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_DOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF_c_xeq_pC_dot_C(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF_c_xeq_pC_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_DOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF_c_xeq_pC_dot_pC(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF_c_xeq_pC_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_DOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF_c_veq_Ca_dot_C(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF_c_veq_Ca_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_ADOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF_c_veq_Ca_dot_pC(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF_c_veq_Ca_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_ADOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF_c_veq_pCa_dot_C(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF_c_veq_pCa_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_ADOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF_c_veq_pCa_dot_pC(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF_c_veq_pCa_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_ADOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF_c_xeq_Ca_dot_C(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF_c_xeq_Ca_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_ADOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF_c_xeq_Ca_dot_pC(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF_c_xeq_Ca_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_ADOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF_c_xeq_pCa_dot_C(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF_c_xeq_pCa_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_ADOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF_c_xeq_pCa_dot_pC(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF_c_xeq_pCa_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_ADOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF_c_veq_sum_C(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF_c_veq_sum_C");
  qlab::api_gsum<float, 1, double>("DF_gsum", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF_c_veq_sum_pC(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF_c_veq_sum_pC");
  qlab::api_gsum<float, 1, double>("DF_gsum", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF_c_xeq_sum_C(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF_c_xeq_sum_C");
  qlab::api_gsum<float, 1, double>("DF_gsum", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF_c_xeq_sum_pC(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF_c_xeq_sum_pC");
  qlab::api_gsum<float, 1, double>("DF_gsum", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DF_r_veq_R_dot_R(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF_r_veq_R_dot_R");
  qlab::api_sred<float, float, qlab::SR_DOT, double>("DF_sred", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF_r_veq_R_dot_pR(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF_r_veq_R_dot_pR");
  qlab::api_sred<float, float, qlab::SR_DOT, double>("DF_sred", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF_r_veq_pR_dot_R(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF_r_veq_pR_dot_R");
  qlab::api_sred<float, float, qlab::SR_DOT, double>("DF_sred", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF_r_veq_pR_dot_pR(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF_r_veq_pR_dot_pR");
  qlab::api_sred<float, float, qlab::SR_DOT, double>("DF_sred", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF_r_xeq_R_dot_R(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF_r_xeq_R_dot_R");
  qlab::api_sred<float, float, qlab::SR_DOT, double>("DF_sred", r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF_r_xeq_R_dot_pR(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF_r_xeq_R_dot_pR");
  qlab::api_sred<float, float, qlab::SR_DOT, double>("DF_sred", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF_r_xeq_pR_dot_R(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF_r_xeq_pR_dot_R");
  qlab::api_sred<float, float, qlab::SR_DOT, double>("DF_sred", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF_r_xeq_pR_dot_pR(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF_r_xeq_pR_dot_pR");
  qlab::api_sred<float, float, qlab::SR_DOT, double>("DF_sred", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF_r_veq_norm2_C(QLA_D_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF_r_veq_norm2_C");
  qlab::api_gdot<float, 1, qlab::LD_NORM2, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DF_r_veq_norm2_pC(QLA_D_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF_r_veq_norm2_pC");
  qlab::api_gdot<float, 1, qlab::LD_NORM2, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DF_r_xeq_norm2_C(QLA_D_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF_r_xeq_norm2_C");
  qlab::api_gdot<float, 1, qlab::LD_NORM2, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DF_r_xeq_norm2_pC(QLA_D_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF_r_xeq_norm2_pC");
  qlab::api_gdot<float, 1, qlab::LD_NORM2, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DF_r_veq_norm2_R(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF_r_veq_norm2_R");
  qlab::api_sred<float, float, qlab::SR_NORM2, double>("DF_sred", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DF_r_veq_norm2_pR(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF_r_veq_norm2_pR");
  qlab::api_sred<float, float, qlab::SR_NORM2, double>("DF_sred", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DF_r_xeq_norm2_R(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF_r_xeq_norm2_R");
  qlab::api_sred<float, float, qlab::SR_NORM2, double>("DF_sred", r, qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DF_r_xeq_norm2_pR(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF_r_xeq_norm2_pR");
  qlab::api_sred<float, float, qlab::SR_NORM2, double>("DF_sred", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DF_r_veq_re_C_dot_C(QLA_D_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF_r_veq_re_C_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_REDOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF_r_veq_re_C_dot_pC(QLA_D_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF_r_veq_re_C_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_REDOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF_r_veq_re_pC_dot_C(QLA_D_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF_r_veq_re_pC_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_REDOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF_r_veq_re_pC_dot_pC(QLA_D_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF_r_veq_re_pC_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_REDOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF_r_xeq_re_C_dot_C(QLA_D_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF_r_xeq_re_C_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_REDOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF_r_xeq_re_C_dot_pC(QLA_D_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, QLA_F_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF_r_xeq_re_C_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_REDOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF_r_xeq_re_pC_dot_C(QLA_D_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF_r_xeq_re_pC_dot_C");
  qlab::api_gdot<float, 1, qlab::LD_REDOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF_r_xeq_re_pC_dot_pC(QLA_D_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, QLA_F_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF_r_xeq_re_pC_dot_pC");
  qlab::api_gdot<float, 1, qlab::LD_REDOT, qlab::PERM_ID, double>("DF_gdot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF_r_veq_sum_R(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF_r_veq_sum_R");
  qlab::api_sred<float, float, qlab::SR_SUM, double>("DF_sred", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DF_r_veq_sum_pR(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF_r_veq_sum_pR");
  qlab::api_sred<float, float, qlab::SR_SUM, double>("DF_sred", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DF_r_xeq_sum_R(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF_r_xeq_sum_R");
  qlab::api_sred<float, float, qlab::SR_SUM, double>("DF_sred", r, qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DF_r_xeq_sum_pR(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF_r_xeq_sum_pR");
  qlab::api_sred<float, float, qlab::SR_SUM, double>("DF_sred", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

}  // extern "C"
