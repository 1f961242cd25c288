// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA DN trace entry points (extern "C"), reference: lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_DN_C_veq_trace_M(int nc, QLA_D_Complex *__restrict__ r, void * a, int n) {
  QLAB_TRACE("QLA_DN_C_veq_trace_M");
  qlab::api_trace_n<double, qlab::SF_TRACE_C>("DN_trace", nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_R_veq_re_trace_M(int nc, QLA_D_Real *__restrict__ r, void * a, int n) {
  QLAB_TRACE("QLA_DN_R_veq_re_trace_M");
  qlab::api_trace_n<double, qlab::SF_TRACE_RE>("DN_trace", nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_R_veq_im_trace_M(int nc, QLA_D_Real *__restrict__ r, void * a, int n) {
  QLAB_TRACE("QLA_DN_R_veq_im_trace_M");
  qlab::api_trace_n<double, qlab::SF_TRACE_IM>("DN_trace", nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_M_veq_antiherm_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_M_veq_antiherm_M");
  qlab::api_antiherm_n<double>("DN_trace", nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_C_veq_trace_pM(int nc, QLA_D_Complex *__restrict__ r, void * a, int n) {
  QLAB_TRACE("QLA_DN_C_veq_trace_pM");
  qlab::api_trace_n<double, qlab::SF_TRACE_C>("DN_trace", nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_R_veq_re_trace_pM(int nc, QLA_D_Real *__restrict__ r, void * a, int n) {
  QLAB_TRACE("QLA_DN_R_veq_re_trace_pM");
  qlab::api_trace_n<double, qlab::SF_TRACE_RE>("DN_trace", nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_R_veq_im_trace_pM(int nc, QLA_D_Real *__restrict__ r, void * a, int n) {
  QLAB_TRACE("QLA_DN_R_veq_im_trace_pM");
  qlab::api_trace_n<double, qlab::SF_TRACE_IM>("DN_trace", nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_M_veq_antiherm_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_M_veq_antiherm_pM");
  qlab::api_antiherm_n<double>("DN_trace", nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_C_xeq_trace_M(int nc, QLA_D_Complex *__restrict__ r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_C_xeq_trace_M");
  qlab::api_trace_n<double, qlab::SF_TRACE_C>("DN_trace", nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DN_R_xeq_re_trace_M(int nc, QLA_D_Real *__restrict__ r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_R_xeq_re_trace_M");
  qlab::api_trace_n<double, qlab::SF_TRACE_RE>("DN_trace", nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DN_R_xeq_im_trace_M(int nc, QLA_D_Real *__restrict__ r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_R_xeq_im_trace_M");
  qlab::api_trace_n<double, qlab::SF_TRACE_IM>("DN_trace", nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DN_M_xeq_antiherm_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeq_antiherm_M");
  qlab::api_antiherm_n<double>("DN_trace", nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DN_C_xeq_trace_pM(int nc, QLA_D_Complex *__restrict__ r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_C_xeq_trace_pM");
  qlab::api_trace_n<double, qlab::SF_TRACE_C>("DN_trace", nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DN_R_xeq_re_trace_pM(int nc, QLA_D_Real *__restrict__ r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_R_xeq_re_trace_pM");
  qlab::api_trace_n<double, qlab::SF_TRACE_RE>("DN_trace", nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DN_R_xeq_im_trace_pM(int nc, QLA_D_Real *__restrict__ r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_R_xeq_im_trace_pM");
  qlab::api_trace_n<double, qlab::SF_TRACE_IM>("DN_trace", nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DN_M_xeq_antiherm_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeq_antiherm_pM");
  qlab::api_antiherm_n<double>("DN_trace", nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

}  // extern "C"
