// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F2 fill entry points (extern "C"), reference: lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_F2_V_veq_v(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_V_veq_v");
  qlab::api_fill_n<float>("F2_fill", 2, 2, r, a, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_v(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_v");
  qlab::api_fill_n<float>("F2_fill", 2, 2, r, a, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_v(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_v");
  qlab::api_fill_n<float>("F2_fill", 2, 2, r, a, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_veqm_v(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_v");
  qlab::api_fill_n<float>("F2_fill", 2, 2, r, a, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veq_zero(QLA_F2_ColorVector *__restrict__ r, int n) {
  QLAB_TRACE("QLA_F2_V_veq_zero");
  qlab::api_zero_n<float>("F2_fill", 2, 2, r, nullptr, n);
}

QLAB_EXPORT void QLA_F2_H_veq_h(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_H_veq_h");
  qlab::api_fill_n<float>("F2_fill", 2, 2 * 2, r, a, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_H_vpeq_h(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_H_vpeq_h");
  qlab::api_fill_n<float>("F2_fill", 2, 2 * 2, r, a, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_H_vmeq_h(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_H_vmeq_h");
  qlab::api_fill_n<float>("F2_fill", 2, 2 * 2, r, a, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_H_veqm_h(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_H_veqm_h");
  qlab::api_fill_n<float>("F2_fill", 2, 2 * 2, r, a, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_H_veq_zero(QLA_F2_HalfFermion *__restrict__ r, int n) {
  QLAB_TRACE("QLA_F2_H_veq_zero");
  qlab::api_zero_n<float>("F2_fill", 2, 2 * 2, r, nullptr, n);
}

QLAB_EXPORT void QLA_F2_D_veq_d(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_D_veq_d");
  qlab::api_fill_n<float>("F2_fill", 2, 4 * 2, r, a, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_D_vpeq_d(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_d");
  qlab::api_fill_n<float>("F2_fill", 2, 4 * 2, r, a, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_D_vmeq_d(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_d");
  qlab::api_fill_n<float>("F2_fill", 2, 4 * 2, r, a, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_D_veqm_d(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_d");
  qlab::api_fill_n<float>("F2_fill", 2, 4 * 2, r, a, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_D_veq_zero(QLA_F2_DiracFermion *__restrict__ r, int n) {
  QLAB_TRACE("QLA_F2_D_veq_zero");
  qlab::api_zero_n<float>("F2_fill", 2, 4 * 2, r, nullptr, n);
}

QLAB_EXPORT void QLA_F2_M_veq_m(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_M_veq_m");
  qlab::api_fill_n<float>("F2_fill", 2, 2 * 2, r, a, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_vpeq_m(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_M_vpeq_m");
  qlab::api_fill_n<float>("F2_fill", 2, 2 * 2, r, a, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_M_vmeq_m(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_M_vmeq_m");
  qlab::api_fill_n<float>("F2_fill", 2, 2 * 2, r, a, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_M_veqm_m(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_M_veqm_m");
  qlab::api_fill_n<float>("F2_fill", 2, 2 * 2, r, a, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_M_veq_zero(QLA_F2_ColorMatrix *__restrict__ r, int n) {
  QLAB_TRACE("QLA_F2_M_veq_zero");
  qlab::api_zero_n<float>("F2_fill", 2, 2 * 2, r, nullptr, n);
}

QLAB_EXPORT void QLA_F2_P_veq_p(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_veq_p");
  qlab::api_fill_n<float>("F2_fill", 2, 16 * 2 * 2, r, a, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_vpeq_p(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_vpeq_p");
  qlab::api_fill_n<float>("F2_fill", 2, 16 * 2 * 2, r, a, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_vmeq_p(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_vmeq_p");
  qlab::api_fill_n<float>("F2_fill", 2, 16 * 2 * 2, r, a, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_veqm_p(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_P_veqm_p");
  qlab::api_fill_n<float>("F2_fill", 2, 16 * 2 * 2, r, a, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_veq_zero(QLA_F2_DiracPropagator *__restrict__ r, int n) {
  QLAB_TRACE("QLA_F2_P_veq_zero");
  qlab::api_zero_n<float>("F2_fill", 2, 16 * 2 * 2, r, nullptr, n);
}

QLAB_EXPORT void QLA_F2_M_veq_c(QLA_F2_ColorMatrix *__restrict__ r, QLA_F_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_M_veq_c");
  qlab::api_diagfill_n<float>("F2_fill", 2, r, a, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_vpeq_c(QLA_F2_ColorMatrix *__restrict__ r, QLA_F_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_M_vpeq_c");
  qlab::api_diagfill_n<float>("F2_fill", 2, r, a, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_M_vmeq_c(QLA_F2_ColorMatrix *__restrict__ r, QLA_F_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_M_vmeq_c");
  qlab::api_diagfill_n<float>("F2_fill", 2, r, a, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_M_veqm_c(QLA_F2_ColorMatrix *__restrict__ r, QLA_F_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_M_veqm_c");
  qlab::api_diagfill_n<float>("F2_fill", 2, r, a, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeq_v(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_v");
  qlab::api_fill_n<float>("F2_fill", 2, 2, r, a, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_v(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_v");
  qlab::api_fill_n<float>("F2_fill", 2, 2, r, a, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_v(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_v");
  qlab::api_fill_n<float>("F2_fill", 2, 2, r, a, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xeqm_v(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_v");
  qlab::api_fill_n<float>("F2_fill", 2, 2, r, a, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeq_zero(QLA_F2_ColorVector *__restrict__ r, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_zero");
  qlab::api_zero_n<float>("F2_fill", 2, 2, r, index, n);
}

QLAB_EXPORT void QLA_F2_H_xeq_h(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_h");
  qlab::api_fill_n<float>("F2_fill", 2, 2 * 2, r, a, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_H_xpeq_h(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xpeq_h");
  qlab::api_fill_n<float>("F2_fill", 2, 2 * 2, r, a, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_H_xmeq_h(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xmeq_h");
  qlab::api_fill_n<float>("F2_fill", 2, 2 * 2, r, a, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_H_xeqm_h(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeqm_h");
  qlab::api_fill_n<float>("F2_fill", 2, 2 * 2, r, a, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_H_xeq_zero(QLA_F2_HalfFermion *__restrict__ r, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_zero");
  qlab::api_zero_n<float>("F2_fill", 2, 2 * 2, r, index, n);
}

QLAB_EXPORT void QLA_F2_D_xeq_d(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_d");
  qlab::api_fill_n<float>("F2_fill", 2, 4 * 2, r, a, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_D_xpeq_d(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_d");
  qlab::api_fill_n<float>("F2_fill", 2, 4 * 2, r, a, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_D_xmeq_d(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_d");
  qlab::api_fill_n<float>("F2_fill", 2, 4 * 2, r, a, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_D_xeqm_d(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_d");
  qlab::api_fill_n<float>("F2_fill", 2, 4 * 2, r, a, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_D_xeq_zero(QLA_F2_DiracFermion *__restrict__ r, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_zero");
  qlab::api_zero_n<float>("F2_fill", 2, 4 * 2, r, index, n);
}

QLAB_EXPORT void QLA_F2_M_xeq_m(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_m");
  qlab::api_fill_n<float>("F2_fill", 2, 2 * 2, r, a, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_xpeq_m(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xpeq_m");
  qlab::api_fill_n<float>("F2_fill", 2, 2 * 2, r, a, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_M_xmeq_m(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xmeq_m");
  qlab::api_fill_n<float>("F2_fill", 2, 2 * 2, r, a, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_M_xeqm_m(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeqm_m");
  qlab::api_fill_n<float>("F2_fill", 2, 2 * 2, r, a, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_M_xeq_zero(QLA_F2_ColorMatrix *__restrict__ r, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_zero");
  qlab::api_zero_n<float>("F2_fill", 2, 2 * 2, r, index, n);
}

QLAB_EXPORT void QLA_F2_P_xeq_p(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_p");
  qlab::api_fill_n<float>("F2_fill", 2, 16 * 2 * 2, r, a, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_P_xpeq_p(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xpeq_p");
  qlab::api_fill_n<float>("F2_fill", 2, 16 * 2 * 2, r, a, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_P_xmeq_p(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xmeq_p");
  qlab::api_fill_n<float>("F2_fill", 2, 16 * 2 * 2, r, a, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_P_xeqm_p(QLA_F2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeqm_p");
  qlab::api_fill_n<float>("F2_fill", 2, 16 * 2 * 2, r, a, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_P_xeq_zero(QLA_F2_DiracPropagator *__restrict__ r, int * index, int n) {
  QLAB_TRACE("QLA_F2_P_xeq_zero");
  qlab::api_zero_n<float>("F2_fill", 2, 16 * 2 * 2, r, index, n);
}

QLAB_EXPORT void QLA_F2_M_xeq_c(QLA_F2_ColorMatrix *__restrict__ r, QLA_F_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_c");
  qlab::api_diagfill_n<float>("F2_fill", 2, r, a, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_xpeq_c(QLA_F2_ColorMatrix *__restrict__ r, QLA_F_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xpeq_c");
  qlab::api_diagfill_n<float>("F2_fill", 2, r, a, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_M_xmeq_c(QLA_F2_ColorMatrix *__restrict__ r, QLA_F_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xmeq_c");
  qlab::api_diagfill_n<float>("F2_fill", 2, r, a, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_M_xeqm_c(QLA_F2_ColorMatrix *__restrict__ r, QLA_F_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeqm_c");
  qlab::api_diagfill_n<float>("F2_fill", 2, r, a, index, n, qlab::EQM);
}

}  // extern "C"
