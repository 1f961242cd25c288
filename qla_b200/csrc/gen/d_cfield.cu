// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA D cfield entry points (extern "C"), reference: lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_scalar.cuh"

extern "C" {
QLAB_EXPORT void QLA_D_C_veq_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_veq_C");
  qlab::api_ew<double, 1, qlab::EW_COPY, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC");
  qlab::api_ew<double, 1, qlab::EW_COPY, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_C");
  qlab::api_ew<double, 1, qlab::EW_COPY, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pC");
  qlab::api_ew<double, 1, qlab::EW_COPY, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_C");
  qlab::api_ew<double, 1, qlab::EW_COPY, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pC");
  qlab::api_ew<double, 1, qlab::EW_COPY, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_veqm_C");
  qlab::api_ew<double, 1, qlab::EW_COPY, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pC");
  qlab::api_ew<double, 1, qlab::EW_COPY, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C");
  qlab::api_ew<double, 1, qlab::EW_COPY, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC");
  qlab::api_ew<double, 1, qlab::EW_COPY, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_C");
  qlab::api_ew<double, 1, qlab::EW_COPY, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pC");
  qlab::api_ew<double, 1, qlab::EW_COPY, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_C");
  qlab::api_ew<double, 1, qlab::EW_COPY, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pC");
  qlab::api_ew<double, 1, qlab::EW_COPY, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_C");
  qlab::api_ew<double, 1, qlab::EW_COPY, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pC");
  qlab::api_ew<double, 1, qlab::EW_COPY, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_veq_Ca");
  qlab::api_ew<double, 1, qlab::EW_CONJ, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_veq_pCa");
  qlab::api_ew<double, 1, qlab::EW_CONJ, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_Ca");
  qlab::api_ew<double, 1, qlab::EW_CONJ, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pCa");
  qlab::api_ew<double, 1, qlab::EW_CONJ, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_Ca");
  qlab::api_ew<double, 1, qlab::EW_CONJ, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pCa");
  qlab::api_ew<double, 1, qlab::EW_CONJ, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_veqm_Ca");
  qlab::api_ew<double, 1, qlab::EW_CONJ, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pCa");
  qlab::api_ew<double, 1, qlab::EW_CONJ, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_Ca");
  qlab::api_ew<double, 1, qlab::EW_CONJ, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pCa");
  qlab::api_ew<double, 1, qlab::EW_CONJ, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_Ca");
  qlab::api_ew<double, 1, qlab::EW_CONJ, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pCa");
  qlab::api_ew<double, 1, qlab::EW_CONJ, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_Ca");
  qlab::api_ew<double, 1, qlab::EW_CONJ, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pCa");
  qlab::api_ew<double, 1, qlab::EW_CONJ, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_Ca");
  qlab::api_ew<double, 1, qlab::EW_CONJ, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pCa");
  qlab::api_ew<double, 1, qlab::EW_CONJ, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_i_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_veq_i_C");
  qlab::api_ew<double, 1, qlab::EW_I, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_i_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_veq_i_pC");
  qlab::api_ew<double, 1, qlab::EW_I, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_i_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_i_C");
  qlab::api_ew<double, 1, qlab::EW_I, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_i_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_i_pC");
  qlab::api_ew<double, 1, qlab::EW_I, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_i_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_i_C");
  qlab::api_ew<double, 1, qlab::EW_I, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_i_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_i_pC");
  qlab::api_ew<double, 1, qlab::EW_I, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_i_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_veqm_i_C");
  qlab::api_ew<double, 1, qlab::EW_I, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_i_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_veqm_i_pC");
  qlab::api_ew<double, 1, qlab::EW_I, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_i_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_i_C");
  qlab::api_ew<double, 1, qlab::EW_I, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_i_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_i_pC");
  qlab::api_ew<double, 1, qlab::EW_I, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_i_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_i_C");
  qlab::api_ew<double, 1, qlab::EW_I, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_i_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_i_pC");
  qlab::api_ew<double, 1, qlab::EW_I, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_i_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_i_C");
  qlab::api_ew<double, 1, qlab::EW_I, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_i_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_i_pC");
  qlab::api_ew<double, 1, qlab::EW_I, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_i_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_i_C");
  qlab::api_ew<double, 1, qlab::EW_I, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_i_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_i_pC");
  qlab::api_ew<double, 1, qlab::EW_I, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_c(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_veq_c");
  qlab::api_fill<double, 1>("D_fill", r, a, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_c(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_c");
  qlab::api_fill<double, 1>("D_fill", r, a, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_c(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_c");
  qlab::api_fill<double, 1>("D_fill", r, a, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_c(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_veqm_c");
  qlab::api_fill<double, 1>("D_fill", r, a, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_c(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_c");
  qlab::api_fill<double, 1>("D_fill", r, a, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_c(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_c");
  qlab::api_fill<double, 1>("D_fill", r, a, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_c(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_c");
  qlab::api_fill<double, 1>("D_fill", r, a, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_c(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_c");
  qlab::api_fill<double, 1>("D_fill", r, a, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_zero(QLA_D_Complex *__restrict__ r, int n) {
  QLAB_TRACE("QLA_D_C_veq_zero");
  qlab::api_zero<double, 1>("D_fill", r, nullptr, n);
}

QLAB_EXPORT void QLA_D_C_xeq_zero(QLA_D_Complex *__restrict__ r, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_zero");
  qlab::api_zero<double, 1>("D_fill", r, index, n);
}

QLAB_EXPORT void QLA_D_C_veq_C_mask_I(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_C_mask_I");
  qlab::api_mask<double, 1>("D_mask", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_D_C_veq_C_mask_pI(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_C_mask_pI");
  qlab::api_mask<double, 1>("D_mask", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_D_C_veq_pC_mask_I(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC_mask_I");
  qlab::api_mask<double, 1>("D_mask", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_D_C_veq_pC_mask_pI(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC_mask_pI");
  qlab::api_mask<double, 1>("D_mask", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_D_C_xeq_C_mask_I(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C_mask_I");
  qlab::api_mask<double, 1>("D_mask", r, qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_D_C_xeq_C_mask_pI(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C_mask_pI");
  qlab::api_mask<double, 1>("D_mask", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_D_C_xeq_pC_mask_I(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC_mask_I");
  qlab::api_mask<double, 1>("D_mask", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_D_C_xeq_pC_mask_pI(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC_mask_pI");
  qlab::api_mask<double, 1>("D_mask", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_D_C_veq_R(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_veq_R");
  qlab::api_scalar<double, qlab::SO_C_FROM_R>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pR(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_veq_pR");
  qlab::api_scalar<double, qlab::SO_C_FROM_R>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_R(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_R");
  qlab::api_scalar<double, qlab::SO_C_FROM_R>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pR(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pR");
  qlab::api_scalar<double, qlab::SO_C_FROM_R>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_R_plus_i_R(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_R_plus_i_R");
  qlab::api_scalar<double, qlab::SO_C_R_PLUS_I_R>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_R_plus_i_pR(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_R_plus_i_pR");
  qlab::api_scalar<double, qlab::SO_C_R_PLUS_I_R>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pR_plus_i_R(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pR_plus_i_R");
  qlab::api_scalar<double, qlab::SO_C_R_PLUS_I_R>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pR_plus_i_pR(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pR_plus_i_pR");
  qlab::api_scalar<double, qlab::SO_C_R_PLUS_I_R>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_R_plus_i_R(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_R_plus_i_R");
  qlab::api_scalar<double, qlab::SO_C_R_PLUS_I_R>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_R_plus_i_pR(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_R_plus_i_pR");
  qlab::api_scalar<double, qlab::SO_C_R_PLUS_I_R>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pR_plus_i_R(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pR_plus_i_R");
  qlab::api_scalar<double, qlab::SO_C_R_PLUS_I_R>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pR_plus_i_pR(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pR_plus_i_pR");
  qlab::api_scalar<double, qlab::SO_C_R_PLUS_I_R>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_C_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_C_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_C_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_C_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pC_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pC_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_C_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_C_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_C_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_C_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pC_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pC_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pC_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pC_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_C_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_C_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_C_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_C_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pC_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pC_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pC_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pC_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_C_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_C_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_C_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_C_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pC_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pC_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pC_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pC_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_C_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_C_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pC_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pC_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_C_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_C_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_C_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_C_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pC_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pC_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pC_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pC_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_C_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_C_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_C_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_C_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pC_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pC_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pC_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pC_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_C_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_C_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_C_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_C_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pC_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pC_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pC_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pC_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_C_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_C_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_C_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_C_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pC_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pC_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_C_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_C_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_C_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_C_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pC_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pC_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pC_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pC_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_C_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_C_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_C_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_C_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pC_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pC_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pC_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pC_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_C_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_C_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_C_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_C_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pC_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pC_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pC_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pC_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_C_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_C_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pC_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pC_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_C_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_C_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_C_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_C_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pC_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pC_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pC_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pC_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_C_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_C_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_C_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_C_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pC_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pC_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pC_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pC_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_C_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_C_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_C_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_C_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pC_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pC_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pC_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pC_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_Ca_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_Ca_times_C");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_Ca_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_Ca_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pCa_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pCa_times_C");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pCa_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pCa_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_Ca_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_Ca_times_C");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_Ca_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_Ca_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pCa_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pCa_times_C");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pCa_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pCa_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_Ca_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_Ca_times_C");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_Ca_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_Ca_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pCa_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pCa_times_C");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pCa_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pCa_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_Ca_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_Ca_times_C");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_Ca_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_Ca_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pCa_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pCa_times_C");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pCa_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pCa_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_Ca_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_Ca_times_C");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_Ca_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_Ca_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pCa_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pCa_times_C");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pCa_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pCa_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_Ca_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_Ca_times_C");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_Ca_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_Ca_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pCa_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pCa_times_C");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pCa_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pCa_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_Ca_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_Ca_times_C");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_Ca_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_Ca_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pCa_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pCa_times_C");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pCa_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pCa_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_Ca_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_Ca_times_C");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_Ca_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_Ca_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pCa_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pCa_times_C");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pCa_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pCa_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CAT, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_Ca_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_Ca_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_Ca_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_Ca_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pCa_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pCa_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pCa_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pCa_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_Ca_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_Ca_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_Ca_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_Ca_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pCa_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pCa_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pCa_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pCa_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_Ca_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_Ca_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_Ca_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_Ca_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pCa_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pCa_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pCa_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pCa_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_Ca_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_Ca_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_Ca_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_Ca_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pCa_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pCa_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pCa_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pCa_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_Ca_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_Ca_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_Ca_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_Ca_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pCa_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pCa_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pCa_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pCa_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_Ca_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_Ca_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_Ca_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_Ca_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pCa_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pCa_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pCa_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pCa_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_Ca_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_Ca_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_Ca_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_Ca_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pCa_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pCa_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pCa_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pCa_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_Ca_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_Ca_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_Ca_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_Ca_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pCa_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pCa_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pCa_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pCa_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CATA, qlab::PERM_ID, qlab::SC_FIELD, false>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_R_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_R_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_R_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_R_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pR_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pR_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pR_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pR_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_R_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_R_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_R_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_R_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pR_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pR_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pR_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pR_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_R_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_R_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_R_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_R_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pR_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pR_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pR_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pR_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_R_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_R_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_R_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_R_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pR_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pR_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pR_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pR_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_R_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_R_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_R_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_R_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pR_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pR_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pR_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pR_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_R_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_R_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_R_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_R_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pR_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pR_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pR_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pR_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_R_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_R_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_R_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_R_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pR_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pR_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pR_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pR_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_R_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_R_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_R_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_R_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pR_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pR_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pR_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pR_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_R_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_R_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_R_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_R_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pR_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pR_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pR_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pR_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_R_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_R_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_R_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_R_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pR_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pR_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pR_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pR_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_R_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_R_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_R_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_R_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pR_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pR_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pR_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pR_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_R_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_R_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_R_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_R_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pR_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pR_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pR_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pR_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_R_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_R_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_R_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_R_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pR_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pR_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pR_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pR_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_R_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_R_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_R_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_R_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pR_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pR_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pR_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pR_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_R_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_R_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_R_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_R_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pR_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pR_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pR_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pR_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_R_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_R_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_R_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_R_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pR_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pR_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pR_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pR_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_FIELD, true>("D_ew", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_c_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_c_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_c_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_c_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_c_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_c_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_c_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_c_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_c_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_c_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_c_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_c_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_c_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_c_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_c_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_c_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_c_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_c_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_c_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_c_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_c_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_c_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_c_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_c_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_c_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_c_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_c_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_c_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_c_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_c_times_C");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_c_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_c_times_pC");
  qlab::api_ew<double, 1, qlab::EW_CT, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_c_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_c_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_c_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_c_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_c_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_c_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_c_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_c_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_c_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_c_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_c_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_c_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_c_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_c_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_c_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_c_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_c_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_c_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_c_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_c_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_c_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_c_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_c_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_c_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_c_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_c_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_c_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_c_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_c_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_c_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_c_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_c_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_CTA, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_r_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_r_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_r_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_r_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_r_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_r_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_r_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_r_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_r_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_r_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_r_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_r_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_r_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_r_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_r_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_r_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_r_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_r_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_r_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_r_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_r_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_r_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_r_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_r_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_r_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_r_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_r_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_r_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_r_times_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_r_times_C");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_r_times_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_r_times_pC");
  qlab::api_ew<double, 1, qlab::EW_RT, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_r_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_r_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_r_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_r_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_r_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_r_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_r_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_r_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_r_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_r_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_r_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_r_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_r_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_r_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_r_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_r_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_r_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_r_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_r_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_r_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_r_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_r_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_r_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_r_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_r_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_r_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_r_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_r_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_r_times_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_r_times_Ca");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_r_times_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_r_times_pCa");
  qlab::api_ew<double, 1, qlab::EW_RTA, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_C_plus_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_C_plus_C");
  qlab::api_ew<double, 1, qlab::EW_PLUS, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_C_plus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_C_plus_pC");
  qlab::api_ew<double, 1, qlab::EW_PLUS, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pC_plus_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC_plus_C");
  qlab::api_ew<double, 1, qlab::EW_PLUS, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pC_plus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC_plus_pC");
  qlab::api_ew<double, 1, qlab::EW_PLUS, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_C_plus_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C_plus_C");
  qlab::api_ew<double, 1, qlab::EW_PLUS, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_C_plus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C_plus_pC");
  qlab::api_ew<double, 1, qlab::EW_PLUS, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pC_plus_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC_plus_C");
  qlab::api_ew<double, 1, qlab::EW_PLUS, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pC_plus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC_plus_pC");
  qlab::api_ew<double, 1, qlab::EW_PLUS, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_C_minus_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_C_minus_C");
  qlab::api_ew<double, 1, qlab::EW_MINUS, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_C_minus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_C_minus_pC");
  qlab::api_ew<double, 1, qlab::EW_MINUS, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pC_minus_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC_minus_C");
  qlab::api_ew<double, 1, qlab::EW_MINUS, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pC_minus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC_minus_pC");
  qlab::api_ew<double, 1, qlab::EW_MINUS, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_C_minus_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C_minus_C");
  qlab::api_ew<double, 1, qlab::EW_MINUS, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_C_minus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C_minus_pC");
  qlab::api_ew<double, 1, qlab::EW_MINUS, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pC_minus_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC_minus_C");
  qlab::api_ew<double, 1, qlab::EW_MINUS, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pC_minus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC_minus_pC");
  qlab::api_ew<double, 1, qlab::EW_MINUS, qlab::PERM_ID, qlab::SC_NONE, false>("D_ew", r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_c_times_C_plus_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, QLA_D_Complex *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D_C_veq_c_times_C_plus_C");
  qlab::api_ew<double, 1, qlab::EW_CT_PLUS, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_c_times_C_plus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, QLA_D_Complex *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D_C_veq_c_times_C_plus_pC");
  qlab::api_ew<double, 1, qlab::EW_CT_PLUS, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_c_times_pC_plus_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, QLA_D_Complex *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D_C_veq_c_times_pC_plus_C");
  qlab::api_ew<double, 1, qlab::EW_CT_PLUS, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_c_times_pC_plus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, QLA_D_Complex *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D_C_veq_c_times_pC_plus_pC");
  qlab::api_ew<double, 1, qlab::EW_CT_PLUS, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_c_times_C_plus_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, QLA_D_Complex *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_c_times_C_plus_C");
  qlab::api_ew<double, 1, qlab::EW_CT_PLUS, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_c_times_C_plus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, QLA_D_Complex *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_c_times_C_plus_pC");
  qlab::api_ew<double, 1, qlab::EW_CT_PLUS, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_c_times_pC_plus_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, QLA_D_Complex *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_c_times_pC_plus_C");
  qlab::api_ew<double, 1, qlab::EW_CT_PLUS, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_c_times_pC_plus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, QLA_D_Complex *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_c_times_pC_plus_pC");
  qlab::api_ew<double, 1, qlab::EW_CT_PLUS, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_c_times_C_minus_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, QLA_D_Complex *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D_C_veq_c_times_C_minus_C");
  qlab::api_ew<double, 1, qlab::EW_CT_MINUS, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_c_times_C_minus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, QLA_D_Complex *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D_C_veq_c_times_C_minus_pC");
  qlab::api_ew<double, 1, qlab::EW_CT_MINUS, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_c_times_pC_minus_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, QLA_D_Complex *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D_C_veq_c_times_pC_minus_C");
  qlab::api_ew<double, 1, qlab::EW_CT_MINUS, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_c_times_pC_minus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, QLA_D_Complex *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D_C_veq_c_times_pC_minus_pC");
  qlab::api_ew<double, 1, qlab::EW_CT_MINUS, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_c_times_C_minus_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, QLA_D_Complex *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_c_times_C_minus_C");
  qlab::api_ew<double, 1, qlab::EW_CT_MINUS, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_c_times_C_minus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, QLA_D_Complex *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_c_times_C_minus_pC");
  qlab::api_ew<double, 1, qlab::EW_CT_MINUS, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_c_times_pC_minus_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, QLA_D_Complex *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_c_times_pC_minus_C");
  qlab::api_ew<double, 1, qlab::EW_CT_MINUS, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_c_times_pC_minus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, QLA_D_Complex *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_c_times_pC_minus_pC");
  qlab::api_ew<double, 1, qlab::EW_CT_MINUS, qlab::PERM_ID, qlab::SC_CONST, false>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_r_times_C_plus_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, QLA_D_Complex *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D_C_veq_r_times_C_plus_C");
  qlab::api_ew<double, 1, qlab::EW_RT_PLUS, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_r_times_C_plus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, QLA_D_Complex *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D_C_veq_r_times_C_plus_pC");
  qlab::api_ew<double, 1, qlab::EW_RT_PLUS, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_r_times_pC_plus_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, QLA_D_Complex *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D_C_veq_r_times_pC_plus_C");
  qlab::api_ew<double, 1, qlab::EW_RT_PLUS, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_r_times_pC_plus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, QLA_D_Complex *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D_C_veq_r_times_pC_plus_pC");
  qlab::api_ew<double, 1, qlab::EW_RT_PLUS, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_r_times_C_plus_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, QLA_D_Complex *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_r_times_C_plus_C");
  qlab::api_ew<double, 1, qlab::EW_RT_PLUS, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_r_times_C_plus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, QLA_D_Complex *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_r_times_C_plus_pC");
  qlab::api_ew<double, 1, qlab::EW_RT_PLUS, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_r_times_pC_plus_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, QLA_D_Complex *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_r_times_pC_plus_C");
  qlab::api_ew<double, 1, qlab::EW_RT_PLUS, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_r_times_pC_plus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, QLA_D_Complex *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_r_times_pC_plus_pC");
  qlab::api_ew<double, 1, qlab::EW_RT_PLUS, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_r_times_C_minus_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, QLA_D_Complex *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D_C_veq_r_times_C_minus_C");
  qlab::api_ew<double, 1, qlab::EW_RT_MINUS, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_r_times_C_minus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, QLA_D_Complex *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D_C_veq_r_times_C_minus_pC");
  qlab::api_ew<double, 1, qlab::EW_RT_MINUS, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_r_times_pC_minus_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, QLA_D_Complex *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D_C_veq_r_times_pC_minus_C");
  qlab::api_ew<double, 1, qlab::EW_RT_MINUS, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_r_times_pC_minus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, QLA_D_Complex *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D_C_veq_r_times_pC_minus_pC");
  qlab::api_ew<double, 1, qlab::EW_RT_MINUS, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_r_times_C_minus_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, QLA_D_Complex *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_r_times_C_minus_C");
  qlab::api_ew<double, 1, qlab::EW_RT_MINUS, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_r_times_C_minus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ b, QLA_D_Complex *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_r_times_C_minus_pC");
  qlab::api_ew<double, 1, qlab::EW_RT_MINUS, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_r_times_pC_minus_C(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, QLA_D_Complex *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_r_times_pC_minus_C");
  qlab::api_ew<double, 1, qlab::EW_RT_MINUS, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_r_times_pC_minus_pC(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D_Complex *__restrict__ * b, QLA_D_Complex *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_r_times_pC_minus_pC");
  qlab::api_ew<double, 1, qlab::EW_RT_MINUS, qlab::PERM_ID, qlab::SC_CONST, true>("D_ew", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_C_divide_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_C_divide_C");
  qlab::api_scalar<double, qlab::SO_C_DIVIDE>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_C_divide_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_C_divide_pC");
  qlab::api_scalar<double, qlab::SO_C_DIVIDE>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pC_divide_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC_divide_C");
  qlab::api_scalar<double, qlab::SO_C_DIVIDE>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pC_divide_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC_divide_pC");
  qlab::api_scalar<double, qlab::SO_C_DIVIDE>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_C_divide_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C_divide_C");
  qlab::api_scalar<double, qlab::SO_C_DIVIDE>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_C_divide_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C_divide_pC");
  qlab::api_scalar<double, qlab::SO_C_DIVIDE>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pC_divide_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC_divide_C");
  qlab::api_scalar<double, qlab::SO_C_DIVIDE>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pC_divide_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC_divide_pC");
  qlab::api_scalar<double, qlab::SO_C_DIVIDE>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_C_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_C_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_C_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_C_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pC_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pC_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_C_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_C_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_C_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_C_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pC_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pC_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pC_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pC_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_C_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_C_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_C_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_C_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pC_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pC_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pC_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pC_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_C_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_C_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_C_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_C_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pC_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pC_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pC_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pC_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_C_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_C_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pC_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pC_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_C_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_C_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_C_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_C_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pC_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pC_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pC_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pC_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_C_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_C_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_C_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_C_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pC_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pC_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pC_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pC_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_C_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_C_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_C_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_C_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pC_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pC_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pC_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pC_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_DOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_C_dot_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_C_dot_Ca");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_C_dot_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_C_dot_pCa");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pC_dot_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC_dot_Ca");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pC_dot_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pC_dot_pCa");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_C_dot_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_C_dot_Ca");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_C_dot_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_C_dot_pCa");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pC_dot_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pC_dot_Ca");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pC_dot_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pC_dot_pCa");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_C_dot_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_C_dot_Ca");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_C_dot_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_C_dot_pCa");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pC_dot_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pC_dot_Ca");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pC_dot_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pC_dot_pCa");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_C_dot_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_C_dot_Ca");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_C_dot_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_C_dot_pCa");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pC_dot_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pC_dot_Ca");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pC_dot_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pC_dot_pCa");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_C_dot_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C_dot_Ca");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_C_dot_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_C_dot_pCa");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pC_dot_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC_dot_Ca");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pC_dot_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pC_dot_pCa");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_C_dot_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_C_dot_Ca");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_C_dot_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_C_dot_pCa");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pC_dot_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pC_dot_Ca");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pC_dot_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pC_dot_pCa");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_C_dot_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_C_dot_Ca");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_C_dot_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_C_dot_pCa");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pC_dot_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pC_dot_Ca");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pC_dot_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pC_dot_pCa");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_C_dot_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_C_dot_Ca");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_C_dot_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_C_dot_pCa");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pC_dot_Ca(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pC_dot_Ca");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pC_dot_pCa(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pC_dot_pCa");
  qlab::api_ldot<double, 1, qlab::LD_DOT_AA, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_Ca_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_Ca_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_Ca_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_Ca_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pCa_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pCa_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_pCa_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veq_pCa_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_Ca_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_Ca_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_Ca_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_Ca_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pCa_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pCa_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vpeq_pCa_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vpeq_pCa_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_Ca_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_Ca_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_Ca_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_Ca_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pCa_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pCa_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_vmeq_pCa_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_vmeq_pCa_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_veqm_Ca_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_Ca_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_Ca_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_Ca_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pCa_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pCa_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veqm_pCa_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_C_veqm_pCa_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeq_Ca_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_Ca_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_Ca_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_Ca_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pCa_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pCa_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_pCa_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_pCa_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_Ca_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_Ca_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_Ca_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_Ca_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pCa_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pCa_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xpeq_pCa_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xpeq_pCa_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_Ca_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_Ca_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_Ca_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_Ca_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pCa_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pCa_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xmeq_pCa_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xmeq_pCa_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_C_xeqm_Ca_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_Ca_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_Ca_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_Ca_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pCa_dot_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pCa_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_xeqm_pCa_dot_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeqm_pCa_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_ADOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_C_veq_cexp_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_veq_cexp_C");
  qlab::api_scalar<double, qlab::SO_C_CEXP>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_cexp_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_veq_cexp_pC");
  qlab::api_scalar<double, qlab::SO_C_CEXP>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_cexp_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_cexp_C");
  qlab::api_scalar<double, qlab::SO_C_CEXP>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_cexp_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_cexp_pC");
  qlab::api_scalar<double, qlab::SO_C_CEXP>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_clog_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_veq_clog_C");
  qlab::api_scalar<double, qlab::SO_C_CLOG>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_clog_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_veq_clog_pC");
  qlab::api_scalar<double, qlab::SO_C_CLOG>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_clog_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_clog_C");
  qlab::api_scalar<double, qlab::SO_C_CLOG>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_clog_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_clog_pC");
  qlab::api_scalar<double, qlab::SO_C_CLOG>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_csqrt_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_veq_csqrt_C");
  qlab::api_scalar<double, qlab::SO_C_CSQRT>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_csqrt_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_veq_csqrt_pC");
  qlab::api_scalar<double, qlab::SO_C_CSQRT>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_csqrt_C(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_csqrt_C");
  qlab::api_scalar<double, qlab::SO_C_CSQRT>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_csqrt_pC(QLA_D_Complex *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_csqrt_pC");
  qlab::api_scalar<double, qlab::SO_C_CSQRT>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_cexpi_R(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_C_veq_cexpi_R");
  qlab::api_scalar<double, qlab::SO_C_CEXPI>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_veq_cexpi_pR(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_C_veq_cexpi_pR");
  qlab::api_scalar<double, qlab::SO_C_CEXPI>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_cexpi_R(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_cexpi_R");
  qlab::api_scalar<double, qlab::SO_C_CEXPI>("D_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_C_xeq_cexpi_pR(QLA_D_Complex *__restrict__ r, QLA_D_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_C_xeq_cexpi_pR");
  qlab::api_scalar<double, qlab::SO_C_CEXPI>("D_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_R_veq_norm2_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_R_veq_norm2_C");
  qlab::api_ldot<double, 1, qlab::LD_NORM2, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_R_veq_norm2_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_R_veq_norm2_pC");
  qlab::api_ldot<double, 1, qlab::LD_NORM2, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_R_vpeq_norm2_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_R_vpeq_norm2_C");
  qlab::api_ldot<double, 1, qlab::LD_NORM2, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_R_vpeq_norm2_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_R_vpeq_norm2_pC");
  qlab::api_ldot<double, 1, qlab::LD_NORM2, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_R_vmeq_norm2_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_R_vmeq_norm2_C");
  qlab::api_ldot<double, 1, qlab::LD_NORM2, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_R_vmeq_norm2_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_R_vmeq_norm2_pC");
  qlab::api_ldot<double, 1, qlab::LD_NORM2, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_R_veqm_norm2_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D_R_veqm_norm2_C");
  qlab::api_ldot<double, 1, qlab::LD_NORM2, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_R_veqm_norm2_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D_R_veqm_norm2_pC");
  qlab::api_ldot<double, 1, qlab::LD_NORM2, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_R_xeq_norm2_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xeq_norm2_C");
  qlab::api_ldot<double, 1, qlab::LD_NORM2, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_R_xeq_norm2_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xeq_norm2_pC");
  qlab::api_ldot<double, 1, qlab::LD_NORM2, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_R_xpeq_norm2_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xpeq_norm2_C");
  qlab::api_ldot<double, 1, qlab::LD_NORM2, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_R_xpeq_norm2_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xpeq_norm2_pC");
  qlab::api_ldot<double, 1, qlab::LD_NORM2, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_R_xmeq_norm2_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xmeq_norm2_C");
  qlab::api_ldot<double, 1, qlab::LD_NORM2, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_R_xmeq_norm2_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xmeq_norm2_pC");
  qlab::api_ldot<double, 1, qlab::LD_NORM2, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_R_xeqm_norm2_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xeqm_norm2_C");
  qlab::api_ldot<double, 1, qlab::LD_NORM2, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_R_xeqm_norm2_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xeqm_norm2_pC");
  qlab::api_ldot<double, 1, qlab::LD_NORM2, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_R_veq_re_C_dot_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_R_veq_re_C_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_R_veq_re_C_dot_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_R_veq_re_C_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_R_veq_re_pC_dot_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_R_veq_re_pC_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_R_veq_re_pC_dot_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_R_veq_re_pC_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_R_vpeq_re_C_dot_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_R_vpeq_re_C_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_R_vpeq_re_C_dot_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_R_vpeq_re_C_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_R_vpeq_re_pC_dot_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_R_vpeq_re_pC_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_R_vpeq_re_pC_dot_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_R_vpeq_re_pC_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_R_vmeq_re_C_dot_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_R_vmeq_re_C_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_R_vmeq_re_C_dot_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_R_vmeq_re_C_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_R_vmeq_re_pC_dot_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_R_vmeq_re_pC_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_R_vmeq_re_pC_dot_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_R_vmeq_re_pC_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_R_veqm_re_C_dot_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_R_veqm_re_C_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_R_veqm_re_C_dot_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_R_veqm_re_C_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_R_veqm_re_pC_dot_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D_R_veqm_re_pC_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_R_veqm_re_pC_dot_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D_R_veqm_re_pC_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_R_xeq_re_C_dot_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xeq_re_C_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_R_xeq_re_C_dot_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xeq_re_C_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_R_xeq_re_pC_dot_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xeq_re_pC_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_R_xeq_re_pC_dot_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xeq_re_pC_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D_R_xpeq_re_C_dot_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xpeq_re_C_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_R_xpeq_re_C_dot_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xpeq_re_C_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_R_xpeq_re_pC_dot_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xpeq_re_pC_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_R_xpeq_re_pC_dot_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xpeq_re_pC_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D_R_xmeq_re_C_dot_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xmeq_re_C_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_R_xmeq_re_C_dot_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xmeq_re_C_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_R_xmeq_re_pC_dot_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xmeq_re_pC_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_R_xmeq_re_pC_dot_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xmeq_re_pC_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D_R_xeqm_re_C_dot_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xeqm_re_C_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_R_xeqm_re_C_dot_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xeqm_re_C_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_R_xeqm_re_pC_dot_C(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xeqm_re_pC_dot_C");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D_R_xeqm_re_pC_dot_pC(QLA_D_Real *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D_Complex *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D_R_xeqm_re_pC_dot_pC");
  qlab::api_ldot<double, 1, qlab::LD_REDOT, qlab::PERM_ID>("D_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

}  // extern "C"
