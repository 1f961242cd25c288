// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA FN random entry points (extern "C"), reference: lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_FN_V_veq_gaussian_S(int nc, void * r, QLA_RandomState *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FN_V_veq_gaussian_S");
  qlab::api_rng_fill_n<float>("FN_random", nc, nc, 1, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FN_V_veq_gaussian_pS(int nc, void * r, QLA_RandomState *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FN_V_veq_gaussian_pS");
  qlab::api_rng_fill_n<float>("FN_random", nc, nc, 1, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FN_H_veq_gaussian_S(int nc, void * r, QLA_RandomState *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FN_H_veq_gaussian_S");
  qlab::api_rng_fill_n<float>("FN_random", nc, 2 * nc, 1, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FN_H_veq_gaussian_pS(int nc, void * r, QLA_RandomState *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FN_H_veq_gaussian_pS");
  qlab::api_rng_fill_n<float>("FN_random", nc, 2 * nc, 1, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FN_D_veq_gaussian_S(int nc, void * r, QLA_RandomState *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FN_D_veq_gaussian_S");
  qlab::api_rng_fill_n<float>("FN_random", nc, 4 * nc, 1, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FN_D_veq_gaussian_pS(int nc, void * r, QLA_RandomState *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FN_D_veq_gaussian_pS");
  qlab::api_rng_fill_n<float>("FN_random", nc, 4 * nc, 1, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FN_M_veq_gaussian_S(int nc, void * r, QLA_RandomState *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_gaussian_S");
  qlab::api_rng_fill_n<float>("FN_random", nc, nc * nc, 1, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FN_M_veq_gaussian_pS(int nc, void * r, QLA_RandomState *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_gaussian_pS");
  qlab::api_rng_fill_n<float>("FN_random", nc, nc * nc, 1, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FN_P_veq_gaussian_S(int nc, void * r, QLA_RandomState *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FN_P_veq_gaussian_S");
  qlab::api_rng_fill_n<float>("FN_random", nc, 16 * nc * nc, 1, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FN_P_veq_gaussian_pS(int nc, void * r, QLA_RandomState *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FN_P_veq_gaussian_pS");
  qlab::api_rng_fill_n<float>("FN_random", nc, 16 * nc * nc, 1, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FN_V_xeq_gaussian_S(int nc, void * r, QLA_RandomState *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_gaussian_S");
  qlab::api_rng_fill_n<float>("FN_random", nc, nc, 1, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FN_V_xeq_gaussian_pS(int nc, void * r, QLA_RandomState *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_gaussian_pS");
  qlab::api_rng_fill_n<float>("FN_random", nc, nc, 1, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FN_H_xeq_gaussian_S(int nc, void * r, QLA_RandomState *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeq_gaussian_S");
  qlab::api_rng_fill_n<float>("FN_random", nc, 2 * nc, 1, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FN_H_xeq_gaussian_pS(int nc, void * r, QLA_RandomState *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeq_gaussian_pS");
  qlab::api_rng_fill_n<float>("FN_random", nc, 2 * nc, 1, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FN_D_xeq_gaussian_S(int nc, void * r, QLA_RandomState *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeq_gaussian_S");
  qlab::api_rng_fill_n<float>("FN_random", nc, 4 * nc, 1, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FN_D_xeq_gaussian_pS(int nc, void * r, QLA_RandomState *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeq_gaussian_pS");
  qlab::api_rng_fill_n<float>("FN_random", nc, 4 * nc, 1, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FN_M_xeq_gaussian_S(int nc, void * r, QLA_RandomState *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_gaussian_S");
  qlab::api_rng_fill_n<float>("FN_random", nc, nc * nc, 1, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FN_M_xeq_gaussian_pS(int nc, void * r, QLA_RandomState *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_gaussian_pS");
  qlab::api_rng_fill_n<float>("FN_random", nc, nc * nc, 1, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FN_P_xeq_gaussian_S(int nc, void * r, QLA_RandomState *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FN_P_xeq_gaussian_S");
  qlab::api_rng_fill_n<float>("FN_random", nc, 16 * nc * nc, 1, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FN_P_xeq_gaussian_pS(int nc, void * r, QLA_RandomState *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_P_xeq_gaussian_pS");
  qlab::api_rng_fill_n<float>("FN_random", nc, 16 * nc * nc, 1, r, qlab::op_ptr((const void* const*)a), index, n);
}

}  // extern "C"
