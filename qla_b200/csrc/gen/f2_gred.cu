// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F2 gred entry points (extern "C"), reference: lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_F2_c_veq_Ma_dot_M(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_Ma_dot_M");
  qlab::api_gdot_n<float, qlab::LD_ADOT, float>("F2_gred", 2, 2 * 2, qlab::PERM_M, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_Ma_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_Ma_dot_pM");
  qlab::api_gdot_n<float, qlab::LD_ADOT, float>("F2_gred", 2, 2 * 2, qlab::PERM_M, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_pMa_dot_M(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_pMa_dot_M");
  qlab::api_gdot_n<float, qlab::LD_ADOT, float>("F2_gred", 2, 2 * 2, qlab::PERM_M, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_pMa_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_pMa_dot_pM");
  qlab::api_gdot_n<float, qlab::LD_ADOT, float>("F2_gred", 2, 2 * 2, qlab::PERM_M, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_P_dot_P(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_P_dot_P");
  qlab::api_gdot_n<float, qlab::LD_DOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_P_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_P_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_DOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_pP_dot_P(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_pP_dot_P");
  qlab::api_gdot_n<float, qlab::LD_DOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_pP_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_pP_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_DOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_Pa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_Pa_dot_P");
  qlab::api_gdot_n<float, qlab::LD_ADOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_P, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_Pa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_Pa_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_ADOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_P, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_pPa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_pPa_dot_P");
  qlab::api_gdot_n<float, qlab::LD_ADOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_P, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_pPa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_pPa_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_ADOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_P, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_P_dot_P(QLA_F_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_P_dot_P");
  qlab::api_gdot_n<float, qlab::LD_REDOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_P_dot_pP(QLA_F_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_P_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_REDOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_pP_dot_P(QLA_F_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_pP_dot_P");
  qlab::api_gdot_n<float, qlab::LD_REDOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_pP_dot_pP(QLA_F_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_pP_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_REDOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_norm2_P(QLA_F_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_r_veq_norm2_P");
  qlab::api_gdot_n<float, qlab::LD_NORM2, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_norm2_pP(QLA_F_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_r_veq_norm2_pP");
  qlab::api_gdot_n<float, qlab::LD_NORM2, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_Ma_dot_M(QLA_D_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_Ma_dot_M");
  qlab::api_gdot_n<float, qlab::LD_ADOT, double>("F2_gred_df", 2, 2 * 2, qlab::PERM_M, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_Ma_dot_pM(QLA_D_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_Ma_dot_pM");
  qlab::api_gdot_n<float, qlab::LD_ADOT, double>("F2_gred_df", 2, 2 * 2, qlab::PERM_M, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_pMa_dot_M(QLA_D_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_pMa_dot_M");
  qlab::api_gdot_n<float, qlab::LD_ADOT, double>("F2_gred_df", 2, 2 * 2, qlab::PERM_M, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_pMa_dot_pM(QLA_D_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_pMa_dot_pM");
  qlab::api_gdot_n<float, qlab::LD_ADOT, double>("F2_gred_df", 2, 2 * 2, qlab::PERM_M, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_P_dot_P(QLA_D_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_P_dot_P");
  qlab::api_gdot_n<float, qlab::LD_DOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_P_dot_pP(QLA_D_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_P_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_DOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_pP_dot_P(QLA_D_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_pP_dot_P");
  qlab::api_gdot_n<float, qlab::LD_DOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_pP_dot_pP(QLA_D_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_pP_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_DOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_Pa_dot_P(QLA_D_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_Pa_dot_P");
  qlab::api_gdot_n<float, qlab::LD_ADOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_P, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_Pa_dot_pP(QLA_D_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_Pa_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_ADOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_P, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_pPa_dot_P(QLA_D_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_pPa_dot_P");
  qlab::api_gdot_n<float, qlab::LD_ADOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_P, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_pPa_dot_pP(QLA_D_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_pPa_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_ADOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_P, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_P_dot_P(QLA_D_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_P_dot_P");
  qlab::api_gdot_n<float, qlab::LD_REDOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_P_dot_pP(QLA_D_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_P_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_REDOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_pP_dot_P(QLA_D_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_pP_dot_P");
  qlab::api_gdot_n<float, qlab::LD_REDOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_pP_dot_pP(QLA_D_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_pP_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_REDOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_norm2_P(QLA_D_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_norm2_P");
  qlab::api_gdot_n<float, qlab::LD_NORM2, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_norm2_pP(QLA_D_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_norm2_pP");
  qlab::api_gdot_n<float, qlab::LD_NORM2, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_Ma_dot_M(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_Ma_dot_M");
  qlab::api_gdot_n<float, qlab::LD_ADOT, float>("F2_gred", 2, 2 * 2, qlab::PERM_M, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_Ma_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_Ma_dot_pM");
  qlab::api_gdot_n<float, qlab::LD_ADOT, float>("F2_gred", 2, 2 * 2, qlab::PERM_M, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_pMa_dot_M(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_pMa_dot_M");
  qlab::api_gdot_n<float, qlab::LD_ADOT, float>("F2_gred", 2, 2 * 2, qlab::PERM_M, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_pMa_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_pMa_dot_pM");
  qlab::api_gdot_n<float, qlab::LD_ADOT, float>("F2_gred", 2, 2 * 2, qlab::PERM_M, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_P_dot_P(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_P_dot_P");
  qlab::api_gdot_n<float, qlab::LD_DOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_P_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_P_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_DOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_pP_dot_P(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_pP_dot_P");
  qlab::api_gdot_n<float, qlab::LD_DOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_pP_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_pP_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_DOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_Pa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_Pa_dot_P");
  qlab::api_gdot_n<float, qlab::LD_ADOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_P, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_Pa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_Pa_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_ADOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_P, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_pPa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_pPa_dot_P");
  qlab::api_gdot_n<float, qlab::LD_ADOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_P, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_pPa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_pPa_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_ADOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_P, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_P_dot_P(QLA_F_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_P_dot_P");
  qlab::api_gdot_n<float, qlab::LD_REDOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_P_dot_pP(QLA_F_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_P_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_REDOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_pP_dot_P(QLA_F_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_pP_dot_P");
  qlab::api_gdot_n<float, qlab::LD_REDOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_pP_dot_pP(QLA_F_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_pP_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_REDOT, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_norm2_P(QLA_F_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_norm2_P");
  qlab::api_gdot_n<float, qlab::LD_NORM2, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_norm2_pP(QLA_F_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_norm2_pP");
  qlab::api_gdot_n<float, qlab::LD_NORM2, float>("F2_gred", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_Ma_dot_M(QLA_D_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_Ma_dot_M");
  qlab::api_gdot_n<float, qlab::LD_ADOT, double>("F2_gred_df", 2, 2 * 2, qlab::PERM_M, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_Ma_dot_pM(QLA_D_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_Ma_dot_pM");
  qlab::api_gdot_n<float, qlab::LD_ADOT, double>("F2_gred_df", 2, 2 * 2, qlab::PERM_M, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_pMa_dot_M(QLA_D_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_pMa_dot_M");
  qlab::api_gdot_n<float, qlab::LD_ADOT, double>("F2_gred_df", 2, 2 * 2, qlab::PERM_M, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_pMa_dot_pM(QLA_D_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_pMa_dot_pM");
  qlab::api_gdot_n<float, qlab::LD_ADOT, double>("F2_gred_df", 2, 2 * 2, qlab::PERM_M, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_P_dot_P(QLA_D_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_P_dot_P");
  qlab::api_gdot_n<float, qlab::LD_DOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_P_dot_pP(QLA_D_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_P_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_DOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_pP_dot_P(QLA_D_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_pP_dot_P");
  qlab::api_gdot_n<float, qlab::LD_DOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_pP_dot_pP(QLA_D_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_pP_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_DOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_Pa_dot_P(QLA_D_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_Pa_dot_P");
  qlab::api_gdot_n<float, qlab::LD_ADOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_P, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_Pa_dot_pP(QLA_D_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_Pa_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_ADOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_P, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_pPa_dot_P(QLA_D_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_pPa_dot_P");
  qlab::api_gdot_n<float, qlab::LD_ADOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_P, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_pPa_dot_pP(QLA_D_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_pPa_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_ADOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_P, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_P_dot_P(QLA_D_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_P_dot_P");
  qlab::api_gdot_n<float, qlab::LD_REDOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_P_dot_pP(QLA_D_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_P_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_REDOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_pP_dot_P(QLA_D_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_pP_dot_P");
  qlab::api_gdot_n<float, qlab::LD_REDOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_pP_dot_pP(QLA_D_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_F2_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_pP_dot_pP");
  qlab::api_gdot_n<float, qlab::LD_REDOT, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_norm2_P(QLA_D_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_norm2_P");
  qlab::api_gdot_n<float, qlab::LD_NORM2, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_norm2_pP(QLA_D_Real *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_norm2_pP");
  qlab::api_gdot_n<float, qlab::LD_NORM2, double>("F2_gred_df", 2, 16 * 2 * 2, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

}  // extern "C"
