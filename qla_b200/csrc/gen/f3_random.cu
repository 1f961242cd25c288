// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F3 random entry points (extern "C"), reference: lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_F3_V_veq_gaussian_S(QLA_F3_ColorVector *__restrict__ r, QLA_RandomState *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_V_veq_gaussian_S");
  qlab::api_rng_fill<float, 3, false>("F3_random", 1, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_V_veq_gaussian_pS(QLA_F3_ColorVector *__restrict__ r, QLA_RandomState *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_V_veq_gaussian_pS");
  qlab::api_rng_fill<float, 3, false>("F3_random", 1, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_H_veq_gaussian_S(QLA_F3_HalfFermion *__restrict__ r, QLA_RandomState *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_H_veq_gaussian_S");
  qlab::api_rng_fill<float, 6, false>("F3_random", 1, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_H_veq_gaussian_pS(QLA_F3_HalfFermion *__restrict__ r, QLA_RandomState *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_H_veq_gaussian_pS");
  qlab::api_rng_fill<float, 6, false>("F3_random", 1, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_D_veq_gaussian_S(QLA_F3_DiracFermion *__restrict__ r, QLA_RandomState *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_D_veq_gaussian_S");
  qlab::api_rng_fill<float, 12, false>("F3_random", 1, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_D_veq_gaussian_pS(QLA_F3_DiracFermion *__restrict__ r, QLA_RandomState *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_D_veq_gaussian_pS");
  qlab::api_rng_fill<float, 12, false>("F3_random", 1, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_M_veq_gaussian_S(QLA_F3_ColorMatrix *__restrict__ r, QLA_RandomState *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_M_veq_gaussian_S");
  qlab::api_rng_fill<float, 9, false>("F3_random", 1, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_M_veq_gaussian_pS(QLA_F3_ColorMatrix *__restrict__ r, QLA_RandomState *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_M_veq_gaussian_pS");
  qlab::api_rng_fill<float, 9, false>("F3_random", 1, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_P_veq_gaussian_S(QLA_F3_DiracPropagator *__restrict__ r, QLA_RandomState *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_P_veq_gaussian_S");
  qlab::api_rng_fill<float, 144, false>("F3_random", 1, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_P_veq_gaussian_pS(QLA_F3_DiracPropagator *__restrict__ r, QLA_RandomState *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_P_veq_gaussian_pS");
  qlab::api_rng_fill<float, 144, false>("F3_random", 1, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_V_xeq_gaussian_S(QLA_F3_ColorVector *__restrict__ r, QLA_RandomState *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_V_xeq_gaussian_S");
  qlab::api_rng_fill<float, 3, false>("F3_random", 1, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_F3_V_xeq_gaussian_pS(QLA_F3_ColorVector *__restrict__ r, QLA_RandomState *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_V_xeq_gaussian_pS");
  qlab::api_rng_fill<float, 3, false>("F3_random", 1, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_F3_H_xeq_gaussian_S(QLA_F3_HalfFermion *__restrict__ r, QLA_RandomState *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_H_xeq_gaussian_S");
  qlab::api_rng_fill<float, 6, false>("F3_random", 1, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_F3_H_xeq_gaussian_pS(QLA_F3_HalfFermion *__restrict__ r, QLA_RandomState *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_H_xeq_gaussian_pS");
  qlab::api_rng_fill<float, 6, false>("F3_random", 1, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_F3_D_xeq_gaussian_S(QLA_F3_DiracFermion *__restrict__ r, QLA_RandomState *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_D_xeq_gaussian_S");
  qlab::api_rng_fill<float, 12, false>("F3_random", 1, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_F3_D_xeq_gaussian_pS(QLA_F3_DiracFermion *__restrict__ r, QLA_RandomState *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_D_xeq_gaussian_pS");
  qlab::api_rng_fill<float, 12, false>("F3_random", 1, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_F3_M_xeq_gaussian_S(QLA_F3_ColorMatrix *__restrict__ r, QLA_RandomState *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xeq_gaussian_S");
  qlab::api_rng_fill<float, 9, false>("F3_random", 1, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_F3_M_xeq_gaussian_pS(QLA_F3_ColorMatrix *__restrict__ r, QLA_RandomState *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xeq_gaussian_pS");
  qlab::api_rng_fill<float, 9, false>("F3_random", 1, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_F3_P_xeq_gaussian_S(QLA_F3_DiracPropagator *__restrict__ r, QLA_RandomState *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_P_xeq_gaussian_S");
  qlab::api_rng_fill<float, 144, false>("F3_random", 1, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_F3_P_xeq_gaussian_pS(QLA_F3_DiracPropagator *__restrict__ r, QLA_RandomState *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_P_xeq_gaussian_pS");
  qlab::api_rng_fill<float, 144, false>("F3_random", 1, r, qlab::op_ptr((const void* const*)a), index, n);
}

}  // extern "C"
