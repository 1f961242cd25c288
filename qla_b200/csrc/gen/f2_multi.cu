// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F2 multi entry points (extern "C"), reference: lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_F2_V_veq_nM_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_veq_nM_times_nV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, false, (const void*)b, false, nullptr, n, nd, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_nM_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ ** b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_veq_nM_times_npV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, false, (const void*)b, true, nullptr, n, nd, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_nMa_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_veq_nMa_times_nV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, false, (const void*)b, false, nullptr, n, nd, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_nMa_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ ** b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_veq_nMa_times_npV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, false, (const void*)b, true, nullptr, n, nd, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_npM_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ * b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_veq_npM_times_nV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, true, (const void*)b, false, nullptr, n, nd, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_npM_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ ** b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_veq_npM_times_npV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, true, (const void*)b, true, nullptr, n, nd, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_npMa_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ * b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_veq_npMa_times_nV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, true, (const void*)b, false, nullptr, n, nd, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_npMa_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ ** b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_veq_npMa_times_npV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, true, (const void*)b, true, nullptr, n, nd, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_nM_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_vpeq_nM_times_nV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, false, (const void*)b, false, nullptr, n, nd, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_nM_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ ** b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_vpeq_nM_times_npV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, false, (const void*)b, true, nullptr, n, nd, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_nMa_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_vpeq_nMa_times_nV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, false, (const void*)b, false, nullptr, n, nd, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_nMa_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ ** b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_vpeq_nMa_times_npV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, false, (const void*)b, true, nullptr, n, nd, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_npM_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ * b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_vpeq_npM_times_nV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, true, (const void*)b, false, nullptr, n, nd, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_npM_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ ** b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_vpeq_npM_times_npV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, true, (const void*)b, true, nullptr, n, nd, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_npMa_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ * b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_vpeq_npMa_times_nV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, true, (const void*)b, false, nullptr, n, nd, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_npMa_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ ** b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_vpeq_npMa_times_npV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, true, (const void*)b, true, nullptr, n, nd, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_nM_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_vmeq_nM_times_nV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, false, (const void*)b, false, nullptr, n, nd, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_nM_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ ** b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_vmeq_nM_times_npV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, false, (const void*)b, true, nullptr, n, nd, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_nMa_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_vmeq_nMa_times_nV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, false, (const void*)b, false, nullptr, n, nd, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_nMa_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ ** b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_vmeq_nMa_times_npV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, false, (const void*)b, true, nullptr, n, nd, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_npM_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ * b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_vmeq_npM_times_nV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, true, (const void*)b, false, nullptr, n, nd, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_npM_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ ** b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_vmeq_npM_times_npV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, true, (const void*)b, true, nullptr, n, nd, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_npMa_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ * b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_vmeq_npMa_times_nV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, true, (const void*)b, false, nullptr, n, nd, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_npMa_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ ** b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_vmeq_npMa_times_npV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, true, (const void*)b, true, nullptr, n, nd, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_veqm_nM_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_veqm_nM_times_nV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, false, (const void*)b, false, nullptr, n, nd, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_nM_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ ** b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_veqm_nM_times_npV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, false, (const void*)b, true, nullptr, n, nd, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_nMa_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_veqm_nMa_times_nV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, false, (const void*)b, false, nullptr, n, nd, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_nMa_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ ** b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_veqm_nMa_times_npV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, false, (const void*)b, true, nullptr, n, nd, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_npM_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ * b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_veqm_npM_times_nV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, true, (const void*)b, false, nullptr, n, nd, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_npM_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ ** b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_veqm_npM_times_npV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, true, (const void*)b, true, nullptr, n, nd, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_npMa_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ * b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_veqm_npMa_times_nV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, true, (const void*)b, false, nullptr, n, nd, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_npMa_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ ** b, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_veqm_npMa_times_npV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, true, (const void*)b, true, nullptr, n, nd, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeq_nM_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xeq_nM_times_nV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, false, (const void*)b, false, index, n, nd, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_nM_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ ** b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xeq_nM_times_npV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, false, (const void*)b, true, index, n, nd, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_nMa_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xeq_nMa_times_nV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, false, (const void*)b, false, index, n, nd, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_nMa_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ ** b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xeq_nMa_times_npV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, false, (const void*)b, true, index, n, nd, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_npM_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xeq_npM_times_nV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, true, (const void*)b, false, index, n, nd, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_npM_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ ** b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xeq_npM_times_npV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, true, (const void*)b, true, index, n, nd, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_npMa_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xeq_npMa_times_nV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, true, (const void*)b, false, index, n, nd, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_npMa_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ ** b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xeq_npMa_times_npV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, true, (const void*)b, true, index, n, nd, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_nM_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xpeq_nM_times_nV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, false, (const void*)b, false, index, n, nd, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_nM_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ ** b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xpeq_nM_times_npV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, false, (const void*)b, true, index, n, nd, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_nMa_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xpeq_nMa_times_nV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, false, (const void*)b, false, index, n, nd, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_nMa_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ ** b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xpeq_nMa_times_npV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, false, (const void*)b, true, index, n, nd, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_npM_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xpeq_npM_times_nV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, true, (const void*)b, false, index, n, nd, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_npM_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ ** b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xpeq_npM_times_npV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, true, (const void*)b, true, index, n, nd, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_npMa_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xpeq_npMa_times_nV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, true, (const void*)b, false, index, n, nd, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_npMa_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ ** b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xpeq_npMa_times_npV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, true, (const void*)b, true, index, n, nd, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_nM_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xmeq_nM_times_nV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, false, (const void*)b, false, index, n, nd, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_nM_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ ** b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xmeq_nM_times_npV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, false, (const void*)b, true, index, n, nd, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_nMa_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xmeq_nMa_times_nV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, false, (const void*)b, false, index, n, nd, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_nMa_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ ** b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xmeq_nMa_times_npV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, false, (const void*)b, true, index, n, nd, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_npM_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xmeq_npM_times_nV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, true, (const void*)b, false, index, n, nd, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_npM_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ ** b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xmeq_npM_times_npV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, true, (const void*)b, true, index, n, nd, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_npMa_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xmeq_npMa_times_nV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, true, (const void*)b, false, index, n, nd, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_npMa_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ ** b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xmeq_npMa_times_npV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, true, (const void*)b, true, index, n, nd, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xeqm_nM_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xeqm_nM_times_nV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, false, (const void*)b, false, index, n, nd, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_nM_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ ** b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xeqm_nM_times_npV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, false, (const void*)b, true, index, n, nd, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_nMa_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xeqm_nMa_times_nV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, false, (const void*)b, false, index, n, nd, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_nMa_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorVector *__restrict__ ** b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xeqm_nMa_times_npV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, false, (const void*)b, true, index, n, nd, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_npM_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xeqm_npM_times_nV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, true, (const void*)b, false, index, n, nd, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_npM_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ ** b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xeqm_npM_times_npV");
  qlab::api_multi_n<float, false>("F2_multi", 2, r, (const void*)a, true, (const void*)b, true, index, n, nd, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_npMa_times_nV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xeqm_npMa_times_nV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, true, (const void*)b, false, index, n, nd, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_npMa_times_npV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ ** a, QLA_F2_ColorVector *__restrict__ ** b, int * index, int n, int nd) {
  QLAB_TRACE("QLA_F2_V_xeqm_npMa_times_npV");
  qlab::api_multi_n<float, true>("F2_multi", 2, r, (const void*)a, true, (const void*)b, true, index, n, nd, qlab::EQM);
}

}  // extern "C"
