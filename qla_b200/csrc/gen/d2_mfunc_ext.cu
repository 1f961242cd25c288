// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA D2 mfunc_ext entry points (extern "C"), reference: lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_mfunc_nc2.cuh"

extern "C" {
QLAB_EXPORT void QLA_D2_M_veq_invsqrt_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_M_veq_invsqrt_M");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_INVSQRT>>("D2_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_veq_log_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_M_veq_log_M");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_LOG>>("D2_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_veq_expA_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_M_veq_expA_M");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EXPA>>("D2_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_veq_expTA_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_M_veq_expTA_M");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EXPTA>>("D2_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_veq_sqrtPH_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_M_veq_sqrtPH_M");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_SQRTPH>>("D2_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_veq_invsqrtPH_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_M_veq_invsqrtPH_M");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_INVSQRTPH>>("D2_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_veq_eigenvals_M(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_V_veq_eigenvals_M");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EIG>>("D2_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_veq_eigenvalsH_M(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_V_veq_eigenvalsH_M");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EIGH>>("D2_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_veq_invsqrt_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_M_veq_invsqrt_pM");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_INVSQRT>>("D2_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_veq_log_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_M_veq_log_pM");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_LOG>>("D2_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_veq_expA_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_M_veq_expA_pM");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EXPA>>("D2_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_veq_expTA_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_M_veq_expTA_pM");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EXPTA>>("D2_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_veq_sqrtPH_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_M_veq_sqrtPH_pM");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_SQRTPH>>("D2_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_veq_invsqrtPH_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_M_veq_invsqrtPH_pM");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_INVSQRTPH>>("D2_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_veq_eigenvals_pM(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_V_veq_eigenvals_pM");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EIG>>("D2_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_veq_eigenvalsH_pM(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_V_veq_eigenvalsH_pM");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EIGH>>("D2_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_veq_M_inverse_V(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, QLA_D2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_V_veq_M_inverse_V");
  qlab::api_map<qlab::Nc2MInverseOp<double, 1>>("D2_minv", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_veq_M_inverse_pV(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, QLA_D2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_V_veq_M_inverse_pV");
  qlab::api_map<qlab::Nc2MInverseOp<double, 1>>("D2_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_veq_pM_inverse_V(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, QLA_D2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_V_veq_pM_inverse_V");
  qlab::api_map<qlab::Nc2MInverseOp<double, 1>>("D2_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_veq_pM_inverse_pV(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, QLA_D2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_V_veq_pM_inverse_pV");
  qlab::api_map<qlab::Nc2MInverseOp<double, 1>>("D2_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_veq_M_inverse_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_M_veq_M_inverse_M");
  qlab::api_map<qlab::Nc2MInverseOp<double, 2>>("D2_minv", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_veq_M_inverse_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_M_veq_M_inverse_pM");
  qlab::api_map<qlab::Nc2MInverseOp<double, 2>>("D2_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_veq_pM_inverse_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, QLA_D2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_M_veq_pM_inverse_M");
  qlab::api_map<qlab::Nc2MInverseOp<double, 2>>("D2_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_veq_pM_inverse_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, QLA_D2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_M_veq_pM_inverse_pM");
  qlab::api_map<qlab::Nc2MInverseOp<double, 2>>("D2_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_invsqrt_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_invsqrt_M");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_INVSQRT>>("D2_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_log_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_log_M");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_LOG>>("D2_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_expA_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_expA_M");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EXPA>>("D2_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_expTA_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_expTA_M");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EXPTA>>("D2_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_sqrtPH_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_sqrtPH_M");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_SQRTPH>>("D2_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_invsqrtPH_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_invsqrtPH_M");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_INVSQRTPH>>("D2_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_xeq_eigenvals_M(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_V_xeq_eigenvals_M");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EIG>>("D2_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_xeq_eigenvalsH_M(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_V_xeq_eigenvalsH_M");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EIGH>>("D2_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_invsqrt_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_invsqrt_pM");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_INVSQRT>>("D2_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_log_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_log_pM");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_LOG>>("D2_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_expA_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_expA_pM");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EXPA>>("D2_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_expTA_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_expTA_pM");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EXPTA>>("D2_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_sqrtPH_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_sqrtPH_pM");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_SQRTPH>>("D2_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_invsqrtPH_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_invsqrtPH_pM");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_INVSQRTPH>>("D2_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_xeq_eigenvals_pM(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_V_xeq_eigenvals_pM");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EIG>>("D2_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_xeq_eigenvalsH_pM(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_V_xeq_eigenvalsH_pM");
  qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EIGH>>("D2_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_xeq_M_inverse_V(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, QLA_D2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_V_xeq_M_inverse_V");
  qlab::api_map<qlab::Nc2MInverseOp<double, 1>>("D2_minv", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_xeq_M_inverse_pV(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, QLA_D2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_V_xeq_M_inverse_pV");
  qlab::api_map<qlab::Nc2MInverseOp<double, 1>>("D2_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_xeq_pM_inverse_V(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, QLA_D2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_V_xeq_pM_inverse_V");
  qlab::api_map<qlab::Nc2MInverseOp<double, 1>>("D2_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_xeq_pM_inverse_pV(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, QLA_D2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_V_xeq_pM_inverse_pV");
  qlab::api_map<qlab::Nc2MInverseOp<double, 1>>("D2_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_M_inverse_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_M_inverse_M");
  qlab::api_map<qlab::Nc2MInverseOp<double, 2>>("D2_minv", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_M_inverse_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_M_inverse_pM");
  qlab::api_map<qlab::Nc2MInverseOp<double, 2>>("D2_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_pM_inverse_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, QLA_D2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_pM_inverse_M");
  qlab::api_map<qlab::Nc2MInverseOp<double, 2>>("D2_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_pM_inverse_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, QLA_D2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_pM_inverse_pM");
  qlab::api_map<qlab::Nc2MInverseOp<double, 2>>("D2_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

}  // extern "C"
