// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA DN gsum entry points (extern "C"), reference: lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_DN_v_veq_sum_V(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_v_veq_sum_V");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_v_veq_sum_pV(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_v_veq_sum_pV");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_h_veq_sum_H(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_h_veq_sum_H");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, 2 * nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_h_veq_sum_pH(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_h_veq_sum_pH");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, 2 * nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_d_veq_sum_D(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_d_veq_sum_D");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, 4 * nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_d_veq_sum_pD(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_d_veq_sum_pD");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, 4 * nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_m_veq_sum_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_m_veq_sum_M");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, nc * nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_m_veq_sum_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_m_veq_sum_pM");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, nc * nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_p_veq_sum_P(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_p_veq_sum_P");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, 16 * nc * nc, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_p_veq_sum_pP(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_p_veq_sum_pP");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, 16 * nc * nc, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DN_v_xeq_sum_V(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_v_xeq_sum_V");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DN_v_xeq_sum_pV(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_v_xeq_sum_pV");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DN_h_xeq_sum_H(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_h_xeq_sum_H");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, 2 * nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DN_h_xeq_sum_pH(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_h_xeq_sum_pH");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, 2 * nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DN_d_xeq_sum_D(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_d_xeq_sum_D");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, 4 * nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DN_d_xeq_sum_pD(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_d_xeq_sum_pD");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, 4 * nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DN_m_xeq_sum_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_m_xeq_sum_M");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, nc * nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DN_m_xeq_sum_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_m_xeq_sum_pM");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, nc * nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DN_p_xeq_sum_P(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_p_xeq_sum_P");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, 16 * nc * nc, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DN_p_xeq_sum_pP(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_p_xeq_sum_pP");
  qlab::api_gsum_n<double, double>("DN_gsum", nc, 16 * nc * nc, r, qlab::op_ptr((const void* const*)a), index, n);
}

}  // extern "C"
