// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA FN convert entry points (extern "C"), reference: lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_DFN_V_veq_V(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_V_veq_V");
  qlab::api_convert_n<float, double>("FN_convert", nc, nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FDN_V_veq_V(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FDN_V_veq_V");
  qlab::api_convert_n<double, float>("FN_convert", nc, nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DFN_V_veq_pV(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_V_veq_pV");
  qlab::api_convert_n<float, double>("FN_convert", nc, nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FDN_V_veq_pV(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FDN_V_veq_pV");
  qlab::api_convert_n<double, float>("FN_convert", nc, nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DFN_H_veq_H(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_H_veq_H");
  qlab::api_convert_n<float, double>("FN_convert", nc, 2 * nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FDN_H_veq_H(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FDN_H_veq_H");
  qlab::api_convert_n<double, float>("FN_convert", nc, 2 * nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DFN_H_veq_pH(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_H_veq_pH");
  qlab::api_convert_n<float, double>("FN_convert", nc, 2 * nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FDN_H_veq_pH(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FDN_H_veq_pH");
  qlab::api_convert_n<double, float>("FN_convert", nc, 2 * nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DFN_D_veq_D(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_D_veq_D");
  qlab::api_convert_n<float, double>("FN_convert", nc, 4 * nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FDN_D_veq_D(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FDN_D_veq_D");
  qlab::api_convert_n<double, float>("FN_convert", nc, 4 * nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DFN_D_veq_pD(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_D_veq_pD");
  qlab::api_convert_n<float, double>("FN_convert", nc, 4 * nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FDN_D_veq_pD(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FDN_D_veq_pD");
  qlab::api_convert_n<double, float>("FN_convert", nc, 4 * nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DFN_M_veq_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_M_veq_M");
  qlab::api_convert_n<float, double>("FN_convert", nc, nc * nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FDN_M_veq_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FDN_M_veq_M");
  qlab::api_convert_n<double, float>("FN_convert", nc, nc * nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DFN_M_veq_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_M_veq_pM");
  qlab::api_convert_n<float, double>("FN_convert", nc, nc * nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FDN_M_veq_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FDN_M_veq_pM");
  qlab::api_convert_n<double, float>("FN_convert", nc, nc * nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DFN_P_veq_P(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_P_veq_P");
  qlab::api_convert_n<float, double>("FN_convert", nc, 16 * nc * nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FDN_P_veq_P(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FDN_P_veq_P");
  qlab::api_convert_n<double, float>("FN_convert", nc, 16 * nc * nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DFN_P_veq_pP(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_P_veq_pP");
  qlab::api_convert_n<float, double>("FN_convert", nc, 16 * nc * nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FDN_P_veq_pP(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FDN_P_veq_pP");
  qlab::api_convert_n<double, float>("FN_convert", nc, 16 * nc * nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DFN_V_xeq_V(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_V_xeq_V");
  qlab::api_convert_n<float, double>("FN_convert", nc, nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FDN_V_xeq_V(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FDN_V_xeq_V");
  qlab::api_convert_n<double, float>("FN_convert", nc, nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DFN_V_xeq_pV(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_V_xeq_pV");
  qlab::api_convert_n<float, double>("FN_convert", nc, nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FDN_V_xeq_pV(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FDN_V_xeq_pV");
  qlab::api_convert_n<double, float>("FN_convert", nc, nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DFN_H_xeq_H(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_H_xeq_H");
  qlab::api_convert_n<float, double>("FN_convert", nc, 2 * nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FDN_H_xeq_H(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FDN_H_xeq_H");
  qlab::api_convert_n<double, float>("FN_convert", nc, 2 * nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DFN_H_xeq_pH(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_H_xeq_pH");
  qlab::api_convert_n<float, double>("FN_convert", nc, 2 * nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FDN_H_xeq_pH(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FDN_H_xeq_pH");
  qlab::api_convert_n<double, float>("FN_convert", nc, 2 * nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DFN_D_xeq_D(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_D_xeq_D");
  qlab::api_convert_n<float, double>("FN_convert", nc, 4 * nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FDN_D_xeq_D(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FDN_D_xeq_D");
  qlab::api_convert_n<double, float>("FN_convert", nc, 4 * nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DFN_D_xeq_pD(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_D_xeq_pD");
  qlab::api_convert_n<float, double>("FN_convert", nc, 4 * nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FDN_D_xeq_pD(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FDN_D_xeq_pD");
  qlab::api_convert_n<double, float>("FN_convert", nc, 4 * nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DFN_M_xeq_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_M_xeq_M");
  qlab::api_convert_n<float, double>("FN_convert", nc, nc * nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FDN_M_xeq_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FDN_M_xeq_M");
  qlab::api_convert_n<double, float>("FN_convert", nc, nc * nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DFN_M_xeq_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_M_xeq_pM");
  qlab::api_convert_n<float, double>("FN_convert", nc, nc * nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FDN_M_xeq_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FDN_M_xeq_pM");
  qlab::api_convert_n<double, float>("FN_convert", nc, nc * nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DFN_P_xeq_P(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_P_xeq_P");
  qlab::api_convert_n<float, double>("FN_convert", nc, 16 * nc * nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FDN_P_xeq_P(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FDN_P_xeq_P");
  qlab::api_convert_n<double, float>("FN_convert", nc, 16 * nc * nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DFN_P_xeq_pP(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_P_xeq_pP");
  qlab::api_convert_n<float, double>("FN_convert", nc, 16 * nc * nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FDN_P_xeq_pP(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FDN_P_xeq_pP");
  qlab::api_convert_n<double, float>("FN_convert", nc, 16 * nc * nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

}  // extern "C"
