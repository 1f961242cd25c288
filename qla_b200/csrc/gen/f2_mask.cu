// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F2 mask entry points (extern "C"), reference: lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_F2_V_veq_V_mask_I(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_V_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 2, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_V_veq_V_mask_pI(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_V_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 2, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_V_veq_pV_mask_I(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_pV_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 2, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_V_veq_pV_mask_pI(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_V_veq_pV_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 2, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_H_veq_H_mask_I(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_H_veq_H_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 2 * 2, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_H_veq_H_mask_pI(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_H_veq_H_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 2 * 2, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_H_veq_pH_mask_I(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_H_veq_pH_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_H_veq_pH_mask_pI(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_H_veq_pH_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_D_veq_D_mask_I(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_D_veq_D_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 4 * 2, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_D_veq_D_mask_pI(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_D_veq_D_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 4 * 2, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_D_veq_pD_mask_I(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_D_veq_pD_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 4 * 2, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_D_veq_pD_mask_pI(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_D_veq_pD_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 4 * 2, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_M_veq_M_mask_I(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_M_veq_M_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 2 * 2, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_M_veq_M_mask_pI(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_M_veq_M_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 2 * 2, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_M_veq_pM_mask_I(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_M_veq_pM_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_M_veq_pM_mask_pI(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_M_veq_pM_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_P_veq_P_mask_I(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_P_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 16 * 2 * 2, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_P_veq_P_mask_pI(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_P_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 16 * 2 * 2, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_P_veq_pP_mask_I(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pP_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 16 * 2 * 2, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_P_veq_pP_mask_pI(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_P_veq_pP_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 16 * 2 * 2, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_V_xeq_V_mask_I(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_V_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 2, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_V_xeq_V_mask_pI(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_V_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 2, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_V_xeq_pV_mask_I(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_pV_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 2, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_V_xeq_pV_mask_pI(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_pV_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 2, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_H_xeq_H_mask_I(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_H_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 2 * 2, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_H_xeq_H_mask_pI(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_H_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 2 * 2, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_H_xeq_pH_mask_I(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_pH_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_H_xeq_pH_mask_pI(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_pH_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_D_xeq_D_mask_I(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_D_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 4 * 2, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_D_xeq_D_mask_pI(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_D_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 4 * 2, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_D_xeq_pD_mask_I(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_pD_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 4 * 2, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_D_xeq_pD_mask_pI(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_pD_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 4 * 2, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_M_xeq_M_mask_I(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_M_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 2 * 2, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_M_xeq_M_mask_pI(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_M_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 2 * 2, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_M_xeq_pM_mask_I(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_pM_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_M_xeq_pM_mask_pI(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_pM_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_P_xeq_P_mask_I(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_P_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 16 * 2 * 2, r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_P_xeq_P_mask_pI(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_P_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 16 * 2 * 2, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_P_xeq_pP_mask_I(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pP_mask_I");
  qlab::api_mask_n<float>("F2_mask", 2, 16 * 2 * 2, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_P_xeq_pP_mask_pI(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_pP_mask_pI");
  qlab::api_mask_n<float>("F2_mask", 2, 16 * 2 * 2, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

}  // extern "C"
