// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA DN fill entry points (extern "C"), reference: lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_DN_V_veq_v(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_V_veq_v");
  qlab::api_fill_n<double>("DN_fill", nc, nc, r, a, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_V_vpeq_v(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_V_vpeq_v");
  qlab::api_fill_n<double>("DN_fill", nc, nc, r, a, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_V_vmeq_v(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_V_vmeq_v");
  qlab::api_fill_n<double>("DN_fill", nc, nc, r, a, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_V_veqm_v(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_V_veqm_v");
  qlab::api_fill_n<double>("DN_fill", nc, nc, r, a, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_V_veq_zero(int nc, void * r, int n) {
  QLAB_TRACE("QLA_DN_V_veq_zero");
  qlab::api_zero_n<double>("DN_fill", nc, nc, r, nullptr, n);
}

QLAB_EXPORT void QLA_DN_H_veq_h(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_H_veq_h");
  qlab::api_fill_n<double>("DN_fill", nc, 2 * nc, r, a, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_H_vpeq_h(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_H_vpeq_h");
  qlab::api_fill_n<double>("DN_fill", nc, 2 * nc, r, a, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_H_vmeq_h(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_H_vmeq_h");
  qlab::api_fill_n<double>("DN_fill", nc, 2 * nc, r, a, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_H_veqm_h(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_H_veqm_h");
  qlab::api_fill_n<double>("DN_fill", nc, 2 * nc, r, a, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_H_veq_zero(int nc, void * r, int n) {
  QLAB_TRACE("QLA_DN_H_veq_zero");
  qlab::api_zero_n<double>("DN_fill", nc, 2 * nc, r, nullptr, n);
}

QLAB_EXPORT void QLA_DN_D_veq_d(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_D_veq_d");
  qlab::api_fill_n<double>("DN_fill", nc, 4 * nc, r, a, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_D_vpeq_d(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_d");
  qlab::api_fill_n<double>("DN_fill", nc, 4 * nc, r, a, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_D_vmeq_d(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_d");
  qlab::api_fill_n<double>("DN_fill", nc, 4 * nc, r, a, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_D_veqm_d(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_d");
  qlab::api_fill_n<double>("DN_fill", nc, 4 * nc, r, a, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_D_veq_zero(int nc, void * r, int n) {
  QLAB_TRACE("QLA_DN_D_veq_zero");
  qlab::api_zero_n<double>("DN_fill", nc, 4 * nc, r, nullptr, n);
}

QLAB_EXPORT void QLA_DN_M_veq_m(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_M_veq_m");
  qlab::api_fill_n<double>("DN_fill", nc, nc * nc, r, a, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_M_vpeq_m(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_M_vpeq_m");
  qlab::api_fill_n<double>("DN_fill", nc, nc * nc, r, a, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_M_vmeq_m(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_M_vmeq_m");
  qlab::api_fill_n<double>("DN_fill", nc, nc * nc, r, a, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_M_veqm_m(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_M_veqm_m");
  qlab::api_fill_n<double>("DN_fill", nc, nc * nc, r, a, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_M_veq_zero(int nc, void * r, int n) {
  QLAB_TRACE("QLA_DN_M_veq_zero");
  qlab::api_zero_n<double>("DN_fill", nc, nc * nc, r, nullptr, n);
}

QLAB_EXPORT void QLA_DN_P_veq_p(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_P_veq_p");
  qlab::api_fill_n<double>("DN_fill", nc, 16 * nc * nc, r, a, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_p(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_p");
  qlab::api_fill_n<double>("DN_fill", nc, 16 * nc * nc, r, a, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_p(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_p");
  qlab::api_fill_n<double>("DN_fill", nc, 16 * nc * nc, r, a, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_veqm_p(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_p");
  qlab::api_fill_n<double>("DN_fill", nc, 16 * nc * nc, r, a, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veq_zero(int nc, void * r, int n) {
  QLAB_TRACE("QLA_DN_P_veq_zero");
  qlab::api_zero_n<double>("DN_fill", nc, 16 * nc * nc, r, nullptr, n);
}

QLAB_EXPORT void QLA_DN_M_veq_c(int nc, void * r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DN_M_veq_c");
  qlab::api_diagfill_n<double>("DN_fill", nc, r, a, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_M_vpeq_c(int nc, void * r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DN_M_vpeq_c");
  qlab::api_diagfill_n<double>("DN_fill", nc, r, a, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_M_vmeq_c(int nc, void * r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DN_M_vmeq_c");
  qlab::api_diagfill_n<double>("DN_fill", nc, r, a, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_M_veqm_c(int nc, void * r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DN_M_veqm_c");
  qlab::api_diagfill_n<double>("DN_fill", nc, r, a, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_V_xeq_v(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_V_xeq_v");
  qlab::api_fill_n<double>("DN_fill", nc, nc, r, a, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_V_xpeq_v(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_V_xpeq_v");
  qlab::api_fill_n<double>("DN_fill", nc, nc, r, a, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_V_xmeq_v(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_V_xmeq_v");
  qlab::api_fill_n<double>("DN_fill", nc, nc, r, a, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_V_xeqm_v(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_V_xeqm_v");
  qlab::api_fill_n<double>("DN_fill", nc, nc, r, a, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_V_xeq_zero(int nc, void * r, int * index, int n) {
  QLAB_TRACE("QLA_DN_V_xeq_zero");
  qlab::api_zero_n<double>("DN_fill", nc, nc, r, index, n);
}

QLAB_EXPORT void QLA_DN_H_xeq_h(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeq_h");
  qlab::api_fill_n<double>("DN_fill", nc, 2 * nc, r, a, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_H_xpeq_h(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xpeq_h");
  qlab::api_fill_n<double>("DN_fill", nc, 2 * nc, r, a, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_H_xmeq_h(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xmeq_h");
  qlab::api_fill_n<double>("DN_fill", nc, 2 * nc, r, a, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_H_xeqm_h(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeqm_h");
  qlab::api_fill_n<double>("DN_fill", nc, 2 * nc, r, a, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_H_xeq_zero(int nc, void * r, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeq_zero");
  qlab::api_zero_n<double>("DN_fill", nc, 2 * nc, r, index, n);
}

QLAB_EXPORT void QLA_DN_D_xeq_d(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_d");
  qlab::api_fill_n<double>("DN_fill", nc, 4 * nc, r, a, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_D_xpeq_d(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_d");
  qlab::api_fill_n<double>("DN_fill", nc, 4 * nc, r, a, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_D_xmeq_d(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_d");
  qlab::api_fill_n<double>("DN_fill", nc, 4 * nc, r, a, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_D_xeqm_d(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_d");
  qlab::api_fill_n<double>("DN_fill", nc, 4 * nc, r, a, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_D_xeq_zero(int nc, void * r, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_zero");
  qlab::api_zero_n<double>("DN_fill", nc, 4 * nc, r, index, n);
}

QLAB_EXPORT void QLA_DN_M_xeq_m(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeq_m");
  qlab::api_fill_n<double>("DN_fill", nc, nc * nc, r, a, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_M_xpeq_m(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xpeq_m");
  qlab::api_fill_n<double>("DN_fill", nc, nc * nc, r, a, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_M_xmeq_m(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xmeq_m");
  qlab::api_fill_n<double>("DN_fill", nc, nc * nc, r, a, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_M_xeqm_m(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeqm_m");
  qlab::api_fill_n<double>("DN_fill", nc, nc * nc, r, a, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_M_xeq_zero(int nc, void * r, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeq_zero");
  qlab::api_zero_n<double>("DN_fill", nc, nc * nc, r, index, n);
}

QLAB_EXPORT void QLA_DN_P_xeq_p(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_p");
  qlab::api_fill_n<double>("DN_fill", nc, 16 * nc * nc, r, a, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_p(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_p");
  qlab::api_fill_n<double>("DN_fill", nc, 16 * nc * nc, r, a, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_p(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_p");
  qlab::api_fill_n<double>("DN_fill", nc, 16 * nc * nc, r, a, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xeqm_p(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_p");
  qlab::api_fill_n<double>("DN_fill", nc, 16 * nc * nc, r, a, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeq_zero(int nc, void * r, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_zero");
  qlab::api_zero_n<double>("DN_fill", nc, 16 * nc * nc, r, index, n);
}

QLAB_EXPORT void QLA_DN_M_xeq_c(int nc, void * r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeq_c");
  qlab::api_diagfill_n<double>("DN_fill", nc, r, a, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_M_xpeq_c(int nc, void * r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xpeq_c");
  qlab::api_diagfill_n<double>("DN_fill", nc, r, a, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_M_xmeq_c(int nc, void * r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xmeq_c");
  qlab::api_diagfill_n<double>("DN_fill", nc, r, a, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_M_xeqm_c(int nc, void * r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeqm_c");
  qlab::api_diagfill_n<double>("DN_fill", nc, r, a, index, n, qlab::EQM);
}

}  // extern "C"
