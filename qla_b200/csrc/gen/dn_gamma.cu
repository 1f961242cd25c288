// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA DN gamma entry points (extern "C"), reference: lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu, mu = 0..15), expressions_gamma.pl:59-134, 384-470
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_DN_D_veq_gamma_times_D(int nc, void * r, void * a, int mu, int n) {
  QLAB_TRACE("QLA_DN_D_veq_gamma_times_D");
  qlab::api_gamma_n<double, true>("DN_gamma", nc, 4 * nc, r, qlab::op_contig(a), mu, nullptr, n);
}

QLAB_EXPORT void QLA_DN_D_veq_gamma_times_pD(int nc, void * r, void * a, int mu, int n) {
  QLAB_TRACE("QLA_DN_D_veq_gamma_times_pD");
  qlab::api_gamma_n<double, true>("DN_gamma", nc, 4 * nc, r, qlab::op_ptr((const void* const*)a), mu, nullptr, n);
}

QLAB_EXPORT void QLA_DN_P_veq_gamma_times_P(int nc, void * r, void * a, int mu, int n) {
  QLAB_TRACE("QLA_DN_P_veq_gamma_times_P");
  qlab::api_gamma_n<double, true>("DN_gamma", nc, 16 * nc * nc, r, qlab::op_contig(a), mu, nullptr, n);
}

QLAB_EXPORT void QLA_DN_P_veq_gamma_times_pP(int nc, void * r, void * a, int mu, int n) {
  QLAB_TRACE("QLA_DN_P_veq_gamma_times_pP");
  qlab::api_gamma_n<double, true>("DN_gamma", nc, 16 * nc * nc, r, qlab::op_ptr((const void* const*)a), mu, nullptr, n);
}

QLAB_EXPORT void QLA_DN_P_veq_P_times_gamma(int nc, void * r, void * a, int mu, int n) {
  QLAB_TRACE("QLA_DN_P_veq_P_times_gamma");
  qlab::api_gamma_n<double, false>("DN_gamma", nc, 16 * nc * nc, r, qlab::op_contig(a), mu, nullptr, n);
}

QLAB_EXPORT void QLA_DN_P_veq_pP_times_gamma(int nc, void * r, void * a, int mu, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pP_times_gamma");
  qlab::api_gamma_n<double, false>("DN_gamma", nc, 16 * nc * nc, r, qlab::op_ptr((const void* const*)a), mu, nullptr, n);
}

QLAB_EXPORT void QLA_DN_D_xeq_gamma_times_D(int nc, void * r, void * a, int mu, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_gamma_times_D");
  qlab::api_gamma_n<double, true>("DN_gamma", nc, 4 * nc, r, qlab::op_contig(a), mu, index, n);
}

QLAB_EXPORT void QLA_DN_D_xeq_gamma_times_pD(int nc, void * r, void * a, int mu, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_gamma_times_pD");
  qlab::api_gamma_n<double, true>("DN_gamma", nc, 4 * nc, r, qlab::op_ptr((const void* const*)a), mu, index, n);
}

QLAB_EXPORT void QLA_DN_P_xeq_gamma_times_P(int nc, void * r, void * a, int mu, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_gamma_times_P");
  qlab::api_gamma_n<double, true>("DN_gamma", nc, 16 * nc * nc, r, qlab::op_contig(a), mu, index, n);
}

QLAB_EXPORT void QLA_DN_P_xeq_gamma_times_pP(int nc, void * r, void * a, int mu, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_gamma_times_pP");
  qlab::api_gamma_n<double, true>("DN_gamma", nc, 16 * nc * nc, r, qlab::op_ptr((const void* const*)a), mu, index, n);
}

QLAB_EXPORT void QLA_DN_P_xeq_P_times_gamma(int nc, void * r, void * a, int mu, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_P_times_gamma");
  qlab::api_gamma_n<double, false>("DN_gamma", nc, 16 * nc * nc, r, qlab::op_contig(a), mu, index, n);
}

QLAB_EXPORT void QLA_DN_P_xeq_pP_times_gamma(int nc, void * r, void * a, int mu, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pP_times_gamma");
  qlab::api_gamma_n<double, false>("DN_gamma", nc, 16 * nc * nc, r, qlab::op_ptr((const void* const*)a), mu, index, n);
}

}  // extern "C"
