// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F random entry points (extern "C"), reference: lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_F_R_veq_random_S(QLA_F_Real *__restrict__ r, QLA_RandomState *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_random_S");
  qlab::api_rng_fill<float, 1, true>("F_random", 0, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_F_R_veq_gaussian_S(QLA_F_Real *__restrict__ r, QLA_RandomState *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_gaussian_S");
  qlab::api_rng_fill<float, 1, true>("F_random", 1, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_F_C_veq_gaussian_S(QLA_F_Complex *__restrict__ r, QLA_RandomState *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_C_veq_gaussian_S");
  qlab::api_rng_fill<float, 1, false>("F_random", 1, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_F_R_veq_random_pS(QLA_F_Real *__restrict__ r, QLA_RandomState *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_random_pS");
  qlab::api_rng_fill<float, 1, true>("F_random", 0, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_F_R_veq_gaussian_pS(QLA_F_Real *__restrict__ r, QLA_RandomState *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_gaussian_pS");
  qlab::api_rng_fill<float, 1, true>("F_random", 1, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_F_C_veq_gaussian_pS(QLA_F_Complex *__restrict__ r, QLA_RandomState *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_C_veq_gaussian_pS");
  qlab::api_rng_fill<float, 1, false>("F_random", 1, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_F_R_xeq_random_S(QLA_F_Real *__restrict__ r, QLA_RandomState *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_random_S");
  qlab::api_rng_fill<float, 1, true>("F_random", 0, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_F_R_xeq_gaussian_S(QLA_F_Real *__restrict__ r, QLA_RandomState *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_gaussian_S");
  qlab::api_rng_fill<float, 1, true>("F_random", 1, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_F_C_xeq_gaussian_S(QLA_F_Complex *__restrict__ r, QLA_RandomState *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_C_xeq_gaussian_S");
  qlab::api_rng_fill<float, 1, false>("F_random", 1, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_F_R_xeq_random_pS(QLA_F_Real *__restrict__ r, QLA_RandomState *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_random_pS");
  qlab::api_rng_fill<float, 1, true>("F_random", 0, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_F_R_xeq_gaussian_pS(QLA_F_Real *__restrict__ r, QLA_RandomState *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_gaussian_pS");
  qlab::api_rng_fill<float, 1, true>("F_random", 1, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_F_C_xeq_gaussian_pS(QLA_F_Complex *__restrict__ r, QLA_RandomState *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_C_xeq_gaussian_pS");
  qlab::api_rng_fill<float, 1, false>("F_random", 1, r, qlab::op_ptr((const void* const*)a), index, n);
}

}  // extern "C"
