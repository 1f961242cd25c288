// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA DN gred entry points (extern "C"), reference: lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_DN_c_veq_Ma_dot_M(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_Ma_dot_M");
  qlab::api_gdot_n<double, qlab::LD_ADOT, double>("DN_gred", nc, nc * nc, qlab::PERM_M, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DN_c_veq_Ma_dot_pM(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_Ma_dot_pM");
  qlab::api_gdot_n<double, qlab::LD_ADOT, double>("DN_gred", nc, nc * nc, qlab::PERM_M, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DN_c_veq_pMa_dot_M(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_pMa_dot_M");
  qlab::api_gdot_n<double, qlab::LD_ADOT, double>("DN_gred", nc, nc * nc, qlab::PERM_M, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DN_c_veq_pMa_dot_pM(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_pMa_dot_pM");
  qlab::api_gdot_n<double, qlab::LD_ADOT, double>("DN_gred", nc, nc * nc, qlab::PERM_M, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DN_c_veq_P_dot_P(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_P_dot_P");
  qlab::api_gdot_n<double, qlab::LD_DOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DN_c_veq_P_dot_pP(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_P_dot_pP");
  qlab::api_gdot_n<double, qlab::LD_DOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DN_c_veq_pP_dot_P(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_pP_dot_P");
  qlab::api_gdot_n<double, qlab::LD_DOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DN_c_veq_pP_dot_pP(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_pP_dot_pP");
  qlab::api_gdot_n<double, qlab::LD_DOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DN_c_veq_Pa_dot_P(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_Pa_dot_P");
  qlab::api_gdot_n<double, qlab::LD_ADOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_P, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DN_c_veq_Pa_dot_pP(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_Pa_dot_pP");
  qlab::api_gdot_n<double, qlab::LD_ADOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_P, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DN_c_veq_pPa_dot_P(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_pPa_dot_P");
  qlab::api_gdot_n<double, qlab::LD_ADOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_P, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DN_c_veq_pPa_dot_pP(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_pPa_dot_pP");
  qlab::api_gdot_n<double, qlab::LD_ADOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_P, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DN_r_veq_re_P_dot_P(int nc, QLA_D_Real *__restrict__ r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_r_veq_re_P_dot_P");
  qlab::api_gdot_n<double, qlab::LD_REDOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DN_r_veq_re_P_dot_pP(int nc, QLA_D_Real *__restrict__ r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_r_veq_re_P_dot_pP");
  qlab::api_gdot_n<double, qlab::LD_REDOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DN_r_veq_re_pP_dot_P(int nc, QLA_D_Real *__restrict__ r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_r_veq_re_pP_dot_P");
  qlab::api_gdot_n<double, qlab::LD_REDOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DN_r_veq_re_pP_dot_pP(int nc, QLA_D_Real *__restrict__ r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_r_veq_re_pP_dot_pP");
  qlab::api_gdot_n<double, qlab::LD_REDOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DN_r_veq_norm2_P(int nc, QLA_D_Real *__restrict__ r, void * a, int n) {
  QLAB_TRACE("QLA_DN_r_veq_norm2_P");
  qlab::api_gdot_n<double, qlab::LD_NORM2, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DN_r_veq_norm2_pP(int nc, QLA_D_Real *__restrict__ r, void * a, int n) {
  QLAB_TRACE("QLA_DN_r_veq_norm2_pP");
  qlab::api_gdot_n<double, qlab::LD_NORM2, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DN_c_xeq_Ma_dot_M(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_Ma_dot_M");
  qlab::api_gdot_n<double, qlab::LD_ADOT, double>("DN_gred", nc, nc * nc, qlab::PERM_M, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DN_c_xeq_Ma_dot_pM(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_Ma_dot_pM");
  qlab::api_gdot_n<double, qlab::LD_ADOT, double>("DN_gred", nc, nc * nc, qlab::PERM_M, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DN_c_xeq_pMa_dot_M(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_pMa_dot_M");
  qlab::api_gdot_n<double, qlab::LD_ADOT, double>("DN_gred", nc, nc * nc, qlab::PERM_M, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DN_c_xeq_pMa_dot_pM(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_pMa_dot_pM");
  qlab::api_gdot_n<double, qlab::LD_ADOT, double>("DN_gred", nc, nc * nc, qlab::PERM_M, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DN_c_xeq_P_dot_P(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_P_dot_P");
  qlab::api_gdot_n<double, qlab::LD_DOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DN_c_xeq_P_dot_pP(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_P_dot_pP");
  qlab::api_gdot_n<double, qlab::LD_DOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DN_c_xeq_pP_dot_P(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_pP_dot_P");
  qlab::api_gdot_n<double, qlab::LD_DOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DN_c_xeq_pP_dot_pP(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_pP_dot_pP");
  qlab::api_gdot_n<double, qlab::LD_DOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DN_c_xeq_Pa_dot_P(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_Pa_dot_P");
  qlab::api_gdot_n<double, qlab::LD_ADOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_P, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DN_c_xeq_Pa_dot_pP(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_Pa_dot_pP");
  qlab::api_gdot_n<double, qlab::LD_ADOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_P, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DN_c_xeq_pPa_dot_P(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_pPa_dot_P");
  qlab::api_gdot_n<double, qlab::LD_ADOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_P, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DN_c_xeq_pPa_dot_pP(int nc, QLA_D_Complex *__restrict__ r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_pPa_dot_pP");
  qlab::api_gdot_n<double, qlab::LD_ADOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_P, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DN_r_xeq_re_P_dot_P(int nc, QLA_D_Real *__restrict__ r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_r_xeq_re_P_dot_P");
  qlab::api_gdot_n<double, qlab::LD_REDOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DN_r_xeq_re_P_dot_pP(int nc, QLA_D_Real *__restrict__ r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_r_xeq_re_P_dot_pP");
  qlab::api_gdot_n<double, qlab::LD_REDOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DN_r_xeq_re_pP_dot_P(int nc, QLA_D_Real *__restrict__ r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_r_xeq_re_pP_dot_P");
  qlab::api_gdot_n<double, qlab::LD_REDOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DN_r_xeq_re_pP_dot_pP(int nc, QLA_D_Real *__restrict__ r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_r_xeq_re_pP_dot_pP");
  qlab::api_gdot_n<double, qlab::LD_REDOT, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DN_r_xeq_norm2_P(int nc, QLA_D_Real *__restrict__ r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_r_xeq_norm2_P");
  qlab::api_gdot_n<double, qlab::LD_NORM2, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DN_r_xeq_norm2_pP(int nc, QLA_D_Real *__restrict__ r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_r_xeq_norm2_pP");
  qlab::api_gdot_n<double, qlab::LD_NORM2, double>("DN_gred", nc, 16 * nc * nc, qlab::PERM_ID, r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

}  // extern "C"
