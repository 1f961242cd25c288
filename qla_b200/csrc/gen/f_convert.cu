// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F convert entry points (extern "C"), reference: lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_scalar.cuh"

extern "C" {
QLAB_EXPORT void QLA_DF_R_veq_R(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF_R_veq_R");
  qlab::api_rconvert<float, double>("DF_convert", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FD_R_veq_R(QLA_F_Real *__restrict__ r, QLA_D_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FD_R_veq_R");
  qlab::api_rconvert<double, float>("DF_convert", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF_R_veq_pR(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF_R_veq_pR");
  qlab::api_rconvert<float, double>("DF_convert", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FD_R_veq_pR(QLA_F_Real *__restrict__ r, QLA_D_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FD_R_veq_pR");
  qlab::api_rconvert<double, float>("DF_convert", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF_C_veq_C(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF_C_veq_C");
  qlab::api_convert<float, double, 1>("DF_convert", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FD_C_veq_C(QLA_F_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FD_C_veq_C");
  qlab::api_convert<double, float, 1>("DF_convert", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF_C_veq_pC(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF_C_veq_pC");
  qlab::api_convert<float, double, 1>("DF_convert", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FD_C_veq_pC(QLA_F_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FD_C_veq_pC");
  qlab::api_convert<double, float, 1>("DF_convert", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF_R_xeq_R(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF_R_xeq_R");
  qlab::api_rconvert<float, double>("DF_convert", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FD_R_xeq_R(QLA_F_Real *__restrict__ r, QLA_D_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FD_R_xeq_R");
  qlab::api_rconvert<double, float>("DF_convert", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF_R_xeq_pR(QLA_D_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF_R_xeq_pR");
  qlab::api_rconvert<float, double>("DF_convert", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FD_R_xeq_pR(QLA_F_Real *__restrict__ r, QLA_D_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FD_R_xeq_pR");
  qlab::api_rconvert<double, float>("DF_convert", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DF_C_xeq_C(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF_C_xeq_C");
  qlab::api_convert<float, double, 1>("DF_convert", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FD_C_xeq_C(QLA_F_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FD_C_xeq_C");
  qlab::api_convert<double, float, 1>("DF_convert", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF_C_xeq_pC(QLA_D_Complex *__restrict__ r, QLA_F_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF_C_xeq_pC");
  qlab::api_convert<float, double, 1>("DF_convert", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FD_C_xeq_pC(QLA_F_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FD_C_xeq_pC");
  qlab::api_convert<double, float, 1>("DF_convert", r, qlab::op_ptr((const void* const*)a), index, n);
}

}  // extern "C"
