// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA I random entry points (extern "C"), reference: lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_S_veq_S(QLA_RandomState *__restrict__ r, QLA_RandomState *__restrict__ a, int n) {
  QLAB_TRACE("QLA_S_veq_S");
  qlab::api_rng_copy("S_state", r, qlab::op_contig(a), qlab::Opnd{}, false, nullptr, n);
}

QLAB_EXPORT void QLA_S_veq_S_mask_I(QLA_RandomState *__restrict__ r, QLA_RandomState *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_S_veq_S_mask_I");
  qlab::api_rng_copy("S_state", r, qlab::op_contig(a), qlab::op_contig(b), true, nullptr, n);
}

QLAB_EXPORT void QLA_S_veq_S_mask_pI(QLA_RandomState *__restrict__ r, QLA_RandomState *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_S_veq_S_mask_pI");
  qlab::api_rng_copy("S_state", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), true, nullptr, n);
}

QLAB_EXPORT void QLA_S_veq_seed_i_I(QLA_RandomState *__restrict__ r, int seed, QLA_Int *__restrict__ a, int n) {
  QLAB_TRACE("QLA_S_veq_seed_i_I");
  qlab::api_rng_seed("S_state", r, seed, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_S_veq_pS(QLA_RandomState *__restrict__ r, QLA_RandomState *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_S_veq_pS");
  qlab::api_rng_copy("S_state", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, false, nullptr, n);
}

QLAB_EXPORT void QLA_S_veq_pS_mask_I(QLA_RandomState *__restrict__ r, QLA_RandomState *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_S_veq_pS_mask_I");
  qlab::api_rng_copy("S_state", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), true, nullptr, n);
}

QLAB_EXPORT void QLA_S_veq_pS_mask_pI(QLA_RandomState *__restrict__ r, QLA_RandomState *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_S_veq_pS_mask_pI");
  qlab::api_rng_copy("S_state", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), true, nullptr, n);
}

QLAB_EXPORT void QLA_S_veq_seed_i_pI(QLA_RandomState *__restrict__ r, int seed, QLA_Int *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_S_veq_seed_i_pI");
  qlab::api_rng_seed("S_state", r, seed, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_S_xeq_S(QLA_RandomState *__restrict__ r, QLA_RandomState *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_S_xeq_S");
  qlab::api_rng_copy("S_state", r, qlab::op_contig(a), qlab::Opnd{}, false, index, n);
}

QLAB_EXPORT void QLA_S_xeq_S_mask_I(QLA_RandomState *__restrict__ r, QLA_RandomState *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_S_xeq_S_mask_I");
  qlab::api_rng_copy("S_state", r, qlab::op_contig(a), qlab::op_contig(b), true, index, n);
}

QLAB_EXPORT void QLA_S_xeq_S_mask_pI(QLA_RandomState *__restrict__ r, QLA_RandomState *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_S_xeq_S_mask_pI");
  qlab::api_rng_copy("S_state", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), true, index, n);
}

QLAB_EXPORT void QLA_S_xeq_seed_i_I(QLA_RandomState *__restrict__ r, int seed, QLA_Int *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_S_xeq_seed_i_I");
  qlab::api_rng_seed("S_state", r, seed, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_S_xeq_pS(QLA_RandomState *__restrict__ r, QLA_RandomState *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_S_xeq_pS");
  qlab::api_rng_copy("S_state", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, false, index, n);
}

QLAB_EXPORT void QLA_S_xeq_pS_mask_I(QLA_RandomState *__restrict__ r, QLA_RandomState *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_S_xeq_pS_mask_I");
  qlab::api_rng_copy("S_state", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), true, index, n);
}

QLAB_EXPORT void QLA_S_xeq_pS_mask_pI(QLA_RandomState *__restrict__ r, QLA_RandomState *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_S_xeq_pS_mask_pI");
  qlab::api_rng_copy("S_state", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), true, index, n);
}

QLAB_EXPORT void QLA_S_xeq_seed_i_pI(QLA_RandomState *__restrict__ r, int seed, QLA_Int *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_S_xeq_seed_i_pI");
  qlab::api_rng_seed("S_state", r, seed, qlab::op_ptr((const void* const*)a), index, n);
}

}  // extern "C"
