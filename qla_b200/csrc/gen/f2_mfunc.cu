// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F2 mfunc entry points (extern "C"), reference: lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_mfunc_nc2.cuh"

extern "C" {
QLAB_EXPORT void QLA_F2_M_veq_exp_M(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_M_veq_exp_M");
  qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EXP>>("F2_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_veq_sqrt_M(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_M_veq_sqrt_M");
  qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_SQRT>>("F2_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_veq_inverse_M(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_M_veq_inverse_M");
  qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_INVERSE>>("F2_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_C_veq_det_M(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_C_veq_det_M");
  qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_DET>>("F2_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_veq_exp_pM(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_M_veq_exp_pM");
  qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EXP>>("F2_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_veq_sqrt_pM(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_M_veq_sqrt_pM");
  qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_SQRT>>("F2_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_veq_inverse_pM(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_M_veq_inverse_pM");
  qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_INVERSE>>("F2_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_C_veq_det_pM(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_C_veq_det_pM");
  qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_DET>>("F2_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_xeq_exp_M(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_exp_M");
  qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EXP>>("F2_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_xeq_sqrt_M(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_sqrt_M");
  qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_SQRT>>("F2_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_xeq_inverse_M(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_inverse_M");
  qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_INVERSE>>("F2_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_C_xeq_det_M(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_C_xeq_det_M");
  qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_DET>>("F2_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_xeq_exp_pM(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_exp_pM");
  qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EXP>>("F2_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_xeq_sqrt_pM(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_sqrt_pM");
  qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_SQRT>>("F2_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_xeq_inverse_pM(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_inverse_pM");
  qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_INVERSE>>("F2_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_C_xeq_det_pM(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_C_xeq_det_pM");
  qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_DET>>("F2_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

}  // extern "C"
