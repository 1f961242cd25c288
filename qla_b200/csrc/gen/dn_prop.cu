// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA DN prop entry points (extern "C"), reference: lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_DN_P_veq_M_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_M_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_M_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_M_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_M_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_M_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_M_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_M_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_Ma_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_Ma_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_Ma_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_Ma_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_Ma_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_Ma_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_Ma_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_Ma_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pM_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pM_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pM_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pM_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pM_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pM_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pM_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pM_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pMa_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pMa_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pMa_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pMa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pMa_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pMa_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pMa_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pMa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_P_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_P_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_P_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_P_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_P_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_P_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_P_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_P_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_P_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_P_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_P_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_P_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_P_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_P_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_P_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_P_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_Pa_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_Pa_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_Pa_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_Pa_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_Pa_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_Pa_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_Pa_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_Pa_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_Pa_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_Pa_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_Pa_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_Pa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_Pa_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_Pa_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_Pa_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_Pa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pP_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pP_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pP_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pP_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pP_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pP_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pP_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pP_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pP_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pP_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pP_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pP_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pP_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pP_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pP_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pP_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pPa_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pPa_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pPa_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pPa_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pPa_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pPa_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pPa_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pPa_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pPa_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pPa_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pPa_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pPa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pPa_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pPa_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_veq_pPa_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veq_pPa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_M_veq_spintrace_P(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_M_veq_spintrace_P");
  qlab::api_prop_n<double, qlab::PK_TRACE, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_M_veq_spintrace_pP(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_M_veq_spintrace_pP");
  qlab::api_prop_n<double, qlab::PK_TRACE, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_M_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_M_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_M_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_M_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_M_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_M_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_M_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_M_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_Ma_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_Ma_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_Ma_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_Ma_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_Ma_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_Ma_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_Ma_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_Ma_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pM_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pM_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pM_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pM_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pM_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pM_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pM_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pM_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pMa_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pMa_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pMa_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pMa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pMa_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pMa_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pMa_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pMa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_P_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_P_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_P_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_P_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_P_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_P_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_P_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_P_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_P_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_P_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_P_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_P_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_P_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_P_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_P_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_P_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_Pa_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_Pa_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_Pa_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_Pa_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_Pa_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_Pa_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_Pa_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_Pa_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_Pa_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_Pa_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_Pa_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_Pa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_Pa_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_Pa_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_Pa_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_Pa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pP_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pP_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pP_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pP_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pP_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pP_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pP_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pP_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pP_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pP_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pP_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pP_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pP_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pP_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pP_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pP_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pPa_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pPa_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pPa_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pPa_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pPa_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pPa_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pPa_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pPa_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pPa_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pPa_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pPa_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pPa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pPa_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pPa_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vpeq_pPa_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vpeq_pPa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_M_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_M_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_M_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_M_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_M_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_M_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_M_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_M_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_Ma_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_Ma_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_Ma_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_Ma_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_Ma_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_Ma_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_Ma_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_Ma_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pM_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pM_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pM_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pM_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pM_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pM_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pM_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pM_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pMa_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pMa_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pMa_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pMa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pMa_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pMa_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pMa_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pMa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_P_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_P_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_P_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_P_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_P_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_P_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_P_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_P_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_P_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_P_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_P_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_P_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_P_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_P_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_P_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_P_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_Pa_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_Pa_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_Pa_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_Pa_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_Pa_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_Pa_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_Pa_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_Pa_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_Pa_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_Pa_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_Pa_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_Pa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_Pa_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_Pa_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_Pa_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_Pa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pP_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pP_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pP_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pP_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pP_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pP_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pP_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pP_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pP_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pP_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pP_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pP_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pP_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pP_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pP_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pP_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pPa_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pPa_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pPa_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pPa_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pPa_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pPa_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pPa_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pPa_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pPa_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pPa_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pPa_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pPa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pPa_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pPa_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_vmeq_pPa_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_vmeq_pPa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_veqm_M_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_M_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_M_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_M_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_M_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_M_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_M_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_M_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_Ma_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_Ma_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_Ma_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_Ma_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_Ma_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_Ma_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_Ma_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_Ma_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pM_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pM_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pM_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pM_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pM_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pM_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pM_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pM_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pMa_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pMa_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pMa_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pMa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pMa_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pMa_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pMa_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pMa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_P_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_P_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_P_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_P_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_P_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_P_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_P_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_P_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_P_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_P_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_P_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_P_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_P_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_P_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_P_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_P_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_Pa_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_Pa_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_Pa_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_Pa_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_Pa_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_Pa_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_Pa_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_Pa_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_Pa_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_Pa_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_Pa_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_Pa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_Pa_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_Pa_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_Pa_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_Pa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pP_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pP_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pP_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pP_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pP_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pP_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pP_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pP_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pP_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pP_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pP_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pP_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pP_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pP_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pP_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pP_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pPa_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pPa_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pPa_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pPa_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pPa_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pPa_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pPa_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pPa_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pPa_times_P(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pPa_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pPa_times_Pa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pPa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pPa_times_pP(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pPa_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_veqm_pPa_times_pPa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_P_veqm_pPa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeq_M_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_M_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_M_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_M_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_M_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_M_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_M_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_M_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_Ma_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_Ma_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_Ma_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_Ma_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_Ma_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_Ma_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_Ma_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_Ma_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pM_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pM_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pM_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pM_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pM_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pM_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pM_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pM_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pMa_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pMa_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pMa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pMa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pMa_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pMa_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pMa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pMa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_P_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_P_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_P_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_P_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_P_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_P_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_P_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_P_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_P_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_P_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_P_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_P_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_P_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_P_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_P_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_P_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_Pa_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_Pa_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_Pa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_Pa_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_Pa_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_Pa_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_Pa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_Pa_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_Pa_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_Pa_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_Pa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_Pa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_Pa_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_Pa_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_Pa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_Pa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pP_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pP_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pP_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pP_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pP_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pP_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pP_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pP_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pP_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pP_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pP_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pP_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pP_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pP_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pP_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pP_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pPa_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pPa_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pPa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pPa_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pPa_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pPa_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pPa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pPa_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pPa_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pPa_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pPa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pPa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pPa_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pPa_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xeq_pPa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeq_pPa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_M_xeq_spintrace_P(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeq_spintrace_P");
  qlab::api_prop_n<double, qlab::PK_TRACE, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_M_xeq_spintrace_pP(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeq_spintrace_pP");
  qlab::api_prop_n<double, qlab::PK_TRACE, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_M_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_M_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_M_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_M_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_M_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_M_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_M_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_M_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_Ma_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_Ma_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_Ma_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_Ma_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_Ma_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_Ma_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_Ma_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_Ma_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pM_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pM_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pM_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pM_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pM_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pM_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pM_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pM_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pMa_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pMa_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pMa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pMa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pMa_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pMa_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pMa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pMa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_P_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_P_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_P_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_P_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_P_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_P_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_P_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_P_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_P_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_P_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_P_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_P_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_P_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_P_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_P_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_P_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_Pa_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_Pa_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_Pa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_Pa_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_Pa_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_Pa_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_Pa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_Pa_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_Pa_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_Pa_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_Pa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_Pa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_Pa_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_Pa_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_Pa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_Pa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pP_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pP_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pP_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pP_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pP_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pP_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pP_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pP_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pP_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pP_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pP_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pP_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pP_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pP_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pP_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pP_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pPa_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pPa_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pPa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pPa_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pPa_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pPa_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pPa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pPa_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pPa_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pPa_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pPa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pPa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pPa_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pPa_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xpeq_pPa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xpeq_pPa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_M_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_M_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_M_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_M_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_M_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_M_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_M_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_M_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_Ma_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_Ma_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_Ma_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_Ma_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_Ma_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_Ma_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_Ma_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_Ma_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pM_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pM_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pM_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pM_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pM_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pM_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pM_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pM_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pMa_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pMa_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pMa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pMa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pMa_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pMa_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pMa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pMa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_P_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_P_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_P_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_P_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_P_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_P_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_P_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_P_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_P_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_P_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_P_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_P_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_P_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_P_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_P_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_P_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_Pa_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_Pa_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_Pa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_Pa_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_Pa_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_Pa_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_Pa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_Pa_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_Pa_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_Pa_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_Pa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_Pa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_Pa_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_Pa_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_Pa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_Pa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pP_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pP_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pP_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pP_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pP_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pP_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pP_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pP_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pP_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pP_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pP_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pP_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pP_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pP_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pP_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pP_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pPa_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pPa_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pPa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pPa_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pPa_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pPa_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pPa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pPa_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pPa_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pPa_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pPa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pPa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pPa_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pPa_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xmeq_pPa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xmeq_pPa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_DN_P_xeqm_M_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_M_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_M_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_M_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_M_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_M_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_M_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_M_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_Ma_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_Ma_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_Ma_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_Ma_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_Ma_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_Ma_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_Ma_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_Ma_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pM_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pM_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pM_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pM_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pM_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pM_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pM_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pM_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pMa_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pMa_times_P");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pMa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pMa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pMa_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pMa_times_pP");
  qlab::api_prop_n<double, qlab::PK_MP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pMa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pMa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_MP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_P_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_P_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_P_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_P_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_P_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_P_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_P_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_P_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_P_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_P_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_P_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_P_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_P_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_P_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_P_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_P_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_Pa_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_Pa_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_Pa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_Pa_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_Pa_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_Pa_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_Pa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_Pa_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_Pa_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_Pa_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_Pa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_Pa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_Pa_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_Pa_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_Pa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_Pa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pP_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pP_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pP_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pP_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pP_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pP_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pP_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pP_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pP_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pP_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pP_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pP_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pP_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pP_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, false, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pP_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pP_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, false, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pPa_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pPa_times_M");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pPa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pPa_times_Ma");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pPa_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pPa_times_pM");
  qlab::api_prop_n<double, qlab::PK_PM, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pPa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pPa_times_pMa");
  qlab::api_prop_n<double, qlab::PK_PM, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pPa_times_P(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pPa_times_P");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pPa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pPa_times_Pa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pPa_times_pP(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pPa_times_pP");
  qlab::api_prop_n<double, qlab::PK_PP, true, false>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_DN_P_xeqm_pPa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_P_xeqm_pPa_times_pPa");
  qlab::api_prop_n<double, qlab::PK_PP, true, true>("DN_prop", nc, r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

}  // extern "C"
