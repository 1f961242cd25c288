// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F2 component entry points (extern "C"), reference: lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_F2_C_veq_elem_V(QLA_F_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int i_c, int n) {
  QLAB_TRACE("QLA_F2_C_veq_elem_V");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'e', 'C', 'V', i_c, 0, 0, 0);
}

QLAB_EXPORT void QLA_F2_V_veq_elem_C(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, int i_c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_elem_C");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'e', 'V', 'C', i_c, 0, 0, 0);
}

QLAB_EXPORT void QLA_F2_C_veq_elem_pV(QLA_F_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int i_c, int n) {
  QLAB_TRACE("QLA_F2_C_veq_elem_pV");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'e', 'C', 'V', i_c, 0, 0, 0);
}

QLAB_EXPORT void QLA_F2_V_veq_elem_pC(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, int i_c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_elem_pC");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'e', 'V', 'C', i_c, 0, 0, 0);
}

QLAB_EXPORT void QLA_F2_C_veq_elem_H(QLA_F_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int i_c, int i_s, int n) {
  QLAB_TRACE("QLA_F2_C_veq_elem_H");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'e', 'C', 'H', i_c, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_H_veq_elem_C(QLA_F2_HalfFermion *__restrict__ r, QLA_F_Complex *__restrict__ a, int i_c, int i_s, int n) {
  QLAB_TRACE("QLA_F2_H_veq_elem_C");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'e', 'H', 'C', i_c, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_C_veq_elem_pH(QLA_F_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, int i_c, int i_s, int n) {
  QLAB_TRACE("QLA_F2_C_veq_elem_pH");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'e', 'C', 'H', i_c, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_H_veq_elem_pC(QLA_F2_HalfFermion *__restrict__ r, QLA_F_Complex *__restrict__ * a, int i_c, int i_s, int n) {
  QLAB_TRACE("QLA_F2_H_veq_elem_pC");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'e', 'H', 'C', i_c, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_C_veq_elem_D(QLA_F_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int i_c, int i_s, int n) {
  QLAB_TRACE("QLA_F2_C_veq_elem_D");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'e', 'C', 'D', i_c, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_D_veq_elem_C(QLA_F2_DiracFermion *__restrict__ r, QLA_F_Complex *__restrict__ a, int i_c, int i_s, int n) {
  QLAB_TRACE("QLA_F2_D_veq_elem_C");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'e', 'D', 'C', i_c, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_C_veq_elem_pD(QLA_F_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int i_c, int i_s, int n) {
  QLAB_TRACE("QLA_F2_C_veq_elem_pD");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'e', 'C', 'D', i_c, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_D_veq_elem_pC(QLA_F2_DiracFermion *__restrict__ r, QLA_F_Complex *__restrict__ * a, int i_c, int i_s, int n) {
  QLAB_TRACE("QLA_F2_D_veq_elem_pC");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'e', 'D', 'C', i_c, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_C_veq_elem_M(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int i_c, int j_c, int n) {
  QLAB_TRACE("QLA_F2_C_veq_elem_M");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'e', 'C', 'M', i_c, 0, j_c, 0);
}

QLAB_EXPORT void QLA_F2_M_veq_elem_C(QLA_F2_ColorMatrix *__restrict__ r, QLA_F_Complex *__restrict__ a, int i_c, int j_c, int n) {
  QLAB_TRACE("QLA_F2_M_veq_elem_C");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'e', 'M', 'C', i_c, 0, j_c, 0);
}

QLAB_EXPORT void QLA_F2_C_veq_elem_pM(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int i_c, int j_c, int n) {
  QLAB_TRACE("QLA_F2_C_veq_elem_pM");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'e', 'C', 'M', i_c, 0, j_c, 0);
}

QLAB_EXPORT void QLA_F2_M_veq_elem_pC(QLA_F2_ColorMatrix *__restrict__ r, QLA_F_Complex *__restrict__ * a, int i_c, int j_c, int n) {
  QLAB_TRACE("QLA_F2_M_veq_elem_pC");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'e', 'M', 'C', i_c, 0, j_c, 0);
}

QLAB_EXPORT void QLA_F2_C_veq_elem_P(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int i_c, int i_s, int j_c, int j_s, int n) {
  QLAB_TRACE("QLA_F2_C_veq_elem_P");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'e', 'C', 'P', i_c, i_s, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_P_veq_elem_C(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, int i_c, int i_s, int j_c, int j_s, int n) {
  QLAB_TRACE("QLA_F2_P_veq_elem_C");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'e', 'P', 'C', i_c, i_s, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_C_veq_elem_pP(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int i_c, int i_s, int j_c, int j_s, int n) {
  QLAB_TRACE("QLA_F2_C_veq_elem_pP");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'e', 'C', 'P', i_c, i_s, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_P_veq_elem_pC(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, int i_c, int i_s, int j_c, int j_s, int n) {
  QLAB_TRACE("QLA_F2_P_veq_elem_pC");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'e', 'P', 'C', i_c, i_s, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_V_veq_colorvec_H(QLA_F2_ColorVector *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int i_s, int n) {
  QLAB_TRACE("QLA_F2_V_veq_colorvec_H");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'c', 'V', 'H', 0, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_H_veq_colorvec_V(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int i_s, int n) {
  QLAB_TRACE("QLA_F2_H_veq_colorvec_V");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'c', 'H', 'V', 0, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_V_veq_colorvec_pH(QLA_F2_ColorVector *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, int i_s, int n) {
  QLAB_TRACE("QLA_F2_V_veq_colorvec_pH");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'c', 'V', 'H', 0, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_H_veq_colorvec_pV(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int i_s, int n) {
  QLAB_TRACE("QLA_F2_H_veq_colorvec_pV");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'c', 'H', 'V', 0, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_V_veq_colorvec_D(QLA_F2_ColorVector *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int i_s, int n) {
  QLAB_TRACE("QLA_F2_V_veq_colorvec_D");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'c', 'V', 'D', 0, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_D_veq_colorvec_V(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int i_s, int n) {
  QLAB_TRACE("QLA_F2_D_veq_colorvec_V");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'c', 'D', 'V', 0, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_V_veq_colorvec_pD(QLA_F2_ColorVector *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int i_s, int n) {
  QLAB_TRACE("QLA_F2_V_veq_colorvec_pD");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'c', 'V', 'D', 0, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_D_veq_colorvec_pV(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int i_s, int n) {
  QLAB_TRACE("QLA_F2_D_veq_colorvec_pV");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'c', 'D', 'V', 0, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_V_veq_colorvec_M(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int j_c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_colorvec_M");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'c', 'V', 'M', 0, 0, j_c, 0);
}

QLAB_EXPORT void QLA_F2_M_veq_colorvec_V(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int j_c, int n) {
  QLAB_TRACE("QLA_F2_M_veq_colorvec_V");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'c', 'M', 'V', 0, 0, j_c, 0);
}

QLAB_EXPORT void QLA_F2_V_veq_colorvec_pM(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int j_c, int n) {
  QLAB_TRACE("QLA_F2_V_veq_colorvec_pM");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'c', 'V', 'M', 0, 0, j_c, 0);
}

QLAB_EXPORT void QLA_F2_M_veq_colorvec_pV(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int j_c, int n) {
  QLAB_TRACE("QLA_F2_M_veq_colorvec_pV");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'c', 'M', 'V', 0, 0, j_c, 0);
}

QLAB_EXPORT void QLA_F2_V_veq_colorvec_P(QLA_F2_ColorVector *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int i_s, int j_c, int j_s, int n) {
  QLAB_TRACE("QLA_F2_V_veq_colorvec_P");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'c', 'V', 'P', 0, i_s, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_P_veq_colorvec_V(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int i_s, int j_c, int j_s, int n) {
  QLAB_TRACE("QLA_F2_P_veq_colorvec_V");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'c', 'P', 'V', 0, i_s, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_V_veq_colorvec_pP(QLA_F2_ColorVector *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int i_s, int j_c, int j_s, int n) {
  QLAB_TRACE("QLA_F2_V_veq_colorvec_pP");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'c', 'V', 'P', 0, i_s, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_P_veq_colorvec_pV(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int i_s, int j_c, int j_s, int n) {
  QLAB_TRACE("QLA_F2_P_veq_colorvec_pV");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'c', 'P', 'V', 0, i_s, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_D_veq_diracvec_P(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int j_c, int j_s, int n) {
  QLAB_TRACE("QLA_F2_D_veq_diracvec_P");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'd', 'D', 'P', 0, 0, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_P_veq_diracvec_D(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int j_c, int j_s, int n) {
  QLAB_TRACE("QLA_F2_P_veq_diracvec_D");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), nullptr, n, 'd', 'P', 'D', 0, 0, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_D_veq_diracvec_pP(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int j_c, int j_s, int n) {
  QLAB_TRACE("QLA_F2_D_veq_diracvec_pP");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'd', 'D', 'P', 0, 0, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_P_veq_diracvec_pD(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int j_c, int j_s, int n) {
  QLAB_TRACE("QLA_F2_P_veq_diracvec_pD");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), nullptr, n, 'd', 'P', 'D', 0, 0, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_C_xeq_elem_V(QLA_F_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int i_c, int * index, int n) {
  QLAB_TRACE("QLA_F2_C_xeq_elem_V");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'e', 'C', 'V', i_c, 0, 0, 0);
}

QLAB_EXPORT void QLA_F2_V_xeq_elem_C(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ a, int i_c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_elem_C");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'e', 'V', 'C', i_c, 0, 0, 0);
}

QLAB_EXPORT void QLA_F2_C_xeq_elem_pV(QLA_F_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int i_c, int * index, int n) {
  QLAB_TRACE("QLA_F2_C_xeq_elem_pV");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'e', 'C', 'V', i_c, 0, 0, 0);
}

QLAB_EXPORT void QLA_F2_V_xeq_elem_pC(QLA_F2_ColorVector *__restrict__ r, QLA_F_Complex *__restrict__ * a, int i_c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_elem_pC");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'e', 'V', 'C', i_c, 0, 0, 0);
}

QLAB_EXPORT void QLA_F2_C_xeq_elem_H(QLA_F_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int i_c, int i_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_C_xeq_elem_H");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'e', 'C', 'H', i_c, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_H_xeq_elem_C(QLA_F2_HalfFermion *__restrict__ r, QLA_F_Complex *__restrict__ a, int i_c, int i_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_elem_C");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'e', 'H', 'C', i_c, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_C_xeq_elem_pH(QLA_F_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, int i_c, int i_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_C_xeq_elem_pH");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'e', 'C', 'H', i_c, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_H_xeq_elem_pC(QLA_F2_HalfFermion *__restrict__ r, QLA_F_Complex *__restrict__ * a, int i_c, int i_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_elem_pC");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'e', 'H', 'C', i_c, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_C_xeq_elem_D(QLA_F_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int i_c, int i_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_C_xeq_elem_D");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'e', 'C', 'D', i_c, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_D_xeq_elem_C(QLA_F2_DiracFermion *__restrict__ r, QLA_F_Complex *__restrict__ a, int i_c, int i_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_elem_C");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'e', 'D', 'C', i_c, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_C_xeq_elem_pD(QLA_F_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int i_c, int i_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_C_xeq_elem_pD");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'e', 'C', 'D', i_c, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_D_xeq_elem_pC(QLA_F2_DiracFermion *__restrict__ r, QLA_F_Complex *__restrict__ * a, int i_c, int i_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_elem_pC");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'e', 'D', 'C', i_c, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_C_xeq_elem_M(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int i_c, int j_c, int * index, int n) {
  QLAB_TRACE("QLA_F2_C_xeq_elem_M");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'e', 'C', 'M', i_c, 0, j_c, 0);
}

QLAB_EXPORT void QLA_F2_M_xeq_elem_C(QLA_F2_ColorMatrix *__restrict__ r, QLA_F_Complex *__restrict__ a, int i_c, int j_c, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_elem_C");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'e', 'M', 'C', i_c, 0, j_c, 0);
}

QLAB_EXPORT void QLA_F2_C_xeq_elem_pM(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int i_c, int j_c, int * index, int n) {
  QLAB_TRACE("QLA_F2_C_xeq_elem_pM");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'e', 'C', 'M', i_c, 0, j_c, 0);
}

QLAB_EXPORT void QLA_F2_M_xeq_elem_pC(QLA_F2_ColorMatrix *__restrict__ r, QLA_F_Complex *__restrict__ * a, int i_c, int j_c, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_elem_pC");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'e', 'M', 'C', i_c, 0, j_c, 0);
}

QLAB_EXPORT void QLA_F2_C_xeq_elem_P(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int i_c, int i_s, int j_c, int j_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_C_xeq_elem_P");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'e', 'C', 'P', i_c, i_s, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_P_xeq_elem_C(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ a, int i_c, int i_s, int j_c, int j_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_elem_C");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'e', 'P', 'C', i_c, i_s, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_C_xeq_elem_pP(QLA_F_Complex *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int i_c, int i_s, int j_c, int j_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_C_xeq_elem_pP");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'e', 'C', 'P', i_c, i_s, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_P_xeq_elem_pC(QLA_F2_DiracPropagator *__restrict__ r, QLA_F_Complex *__restrict__ * a, int i_c, int i_s, int j_c, int j_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_elem_pC");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'e', 'P', 'C', i_c, i_s, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_V_xeq_colorvec_H(QLA_F2_ColorVector *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int i_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_colorvec_H");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'c', 'V', 'H', 0, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_H_xeq_colorvec_V(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int i_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_colorvec_V");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'c', 'H', 'V', 0, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_V_xeq_colorvec_pH(QLA_F2_ColorVector *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, int i_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_colorvec_pH");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'c', 'V', 'H', 0, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_H_xeq_colorvec_pV(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int i_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_colorvec_pV");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'c', 'H', 'V', 0, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_V_xeq_colorvec_D(QLA_F2_ColorVector *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int i_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_colorvec_D");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'c', 'V', 'D', 0, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_D_xeq_colorvec_V(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int i_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_colorvec_V");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'c', 'D', 'V', 0, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_V_xeq_colorvec_pD(QLA_F2_ColorVector *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int i_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_colorvec_pD");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'c', 'V', 'D', 0, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_D_xeq_colorvec_pV(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int i_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_colorvec_pV");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'c', 'D', 'V', 0, i_s, 0, 0);
}

QLAB_EXPORT void QLA_F2_V_xeq_colorvec_M(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int j_c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_colorvec_M");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'c', 'V', 'M', 0, 0, j_c, 0);
}

QLAB_EXPORT void QLA_F2_M_xeq_colorvec_V(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int j_c, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_colorvec_V");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'c', 'M', 'V', 0, 0, j_c, 0);
}

QLAB_EXPORT void QLA_F2_V_xeq_colorvec_pM(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int j_c, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_colorvec_pM");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'c', 'V', 'M', 0, 0, j_c, 0);
}

QLAB_EXPORT void QLA_F2_M_xeq_colorvec_pV(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int j_c, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_colorvec_pV");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'c', 'M', 'V', 0, 0, j_c, 0);
}

QLAB_EXPORT void QLA_F2_V_xeq_colorvec_P(QLA_F2_ColorVector *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int i_s, int j_c, int j_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_colorvec_P");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'c', 'V', 'P', 0, i_s, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_P_xeq_colorvec_V(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int i_s, int j_c, int j_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_colorvec_V");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'c', 'P', 'V', 0, i_s, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_V_xeq_colorvec_pP(QLA_F2_ColorVector *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int i_s, int j_c, int j_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_colorvec_pP");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'c', 'V', 'P', 0, i_s, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_P_xeq_colorvec_pV(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int i_s, int j_c, int j_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_colorvec_pV");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'c', 'P', 'V', 0, i_s, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_D_xeq_diracvec_P(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int j_c, int j_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_diracvec_P");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'd', 'D', 'P', 0, 0, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_P_xeq_diracvec_D(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int j_c, int j_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_diracvec_D");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_contig(a), index, n, 'd', 'P', 'D', 0, 0, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_D_xeq_diracvec_pP(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int j_c, int j_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_diracvec_pP");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'd', 'D', 'P', 0, 0, j_c, j_s);
}

QLAB_EXPORT void QLA_F2_P_xeq_diracvec_pD(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int j_c, int j_s, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_diracvec_pD");
  qlab::api_sub_n<float>("F2_component", 2, r, qlab::op_ptr((const void* const*)a), index, n, 'd', 'P', 'D', 0, 0, j_c, j_s);
}

}  // extern "C"
