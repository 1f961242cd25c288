// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F3 ldot entry points (extern "C"), reference: lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ewise.cuh"

extern "C" {
QLAB_EXPORT void QLA_F3_C_veq_V_dot_V(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_V_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_V_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_V_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_V_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_V_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_V_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_V_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pV_dot_V(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pV_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_pV_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_pV_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pV_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pV_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_pV_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_pV_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_norm2_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_veq_norm2_V");
  qlab::api_ldot<float, 3, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_norm2_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_veq_norm2_pV");
  qlab::api_ldot<float, 3, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_V_dot_V(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_V_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_V_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_V_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_V_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_V_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_V_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_V_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pV_dot_V(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pV_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_pV_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_pV_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pV_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pV_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_pV_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_pV_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_norm2_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_norm2_V");
  qlab::api_ldot<float, 3, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_norm2_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_norm2_pV");
  qlab::api_ldot<float, 3, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_V_dot_V(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_V_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_V_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_V_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_V_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_V_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_V_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_V_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pV_dot_V(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pV_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_pV_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_pV_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pV_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pV_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_pV_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_pV_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_norm2_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_norm2_V");
  qlab::api_ldot<float, 3, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_norm2_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_norm2_pV");
  qlab::api_ldot<float, 3, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_veqm_V_dot_V(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_V_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_V_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_V_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_V_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_V_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_V_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_V_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pV_dot_V(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pV_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_pV_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_pV_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pV_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pV_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_pV_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_pV_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_norm2_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_norm2_V");
  qlab::api_ldot<float, 3, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_norm2_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_norm2_pV");
  qlab::api_ldot<float, 3, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeq_V_dot_V(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_V_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_V_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_V_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_V_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_V_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_V_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_V_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pV_dot_V(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pV_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_pV_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_pV_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pV_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pV_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_pV_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_pV_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_norm2_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_norm2_V");
  qlab::api_ldot<float, 3, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_norm2_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_norm2_pV");
  qlab::api_ldot<float, 3, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_V_dot_V(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_V_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_V_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_V_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_V_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_V_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_V_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_V_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pV_dot_V(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pV_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_pV_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_pV_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pV_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pV_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_pV_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_pV_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_norm2_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_norm2_V");
  qlab::api_ldot<float, 3, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_norm2_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_norm2_pV");
  qlab::api_ldot<float, 3, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_V_dot_V(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_V_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_V_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_V_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_V_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_V_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_V_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_V_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pV_dot_V(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pV_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_pV_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_pV_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pV_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pV_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_pV_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_pV_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_norm2_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_norm2_V");
  qlab::api_ldot<float, 3, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_norm2_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_norm2_pV");
  qlab::api_ldot<float, 3, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xeqm_V_dot_V(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_V_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_V_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_V_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_V_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_V_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_V_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_V_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pV_dot_V(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pV_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_pV_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_pV_dot_V");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pV_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pV_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_pV_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_pV_dot_pV");
  qlab::api_ldot<float, 3, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_norm2_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_norm2_V");
  qlab::api_ldot<float, 3, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_norm2_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_norm2_pV");
  qlab::api_ldot<float, 3, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veq_H_dot_H(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_H_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_H_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_H_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_H_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_H_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_H_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_H_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pH_dot_H(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pH_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_pH_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_pH_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pH_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pH_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_pH_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_pH_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_norm2_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_veq_norm2_H");
  qlab::api_ldot<float, 6, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_norm2_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_veq_norm2_pH");
  qlab::api_ldot<float, 6, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_H_dot_H(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_H_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_H_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_H_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_H_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_H_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_H_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_H_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pH_dot_H(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pH_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_pH_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_pH_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pH_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pH_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_pH_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_pH_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_norm2_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_norm2_H");
  qlab::api_ldot<float, 6, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_norm2_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_norm2_pH");
  qlab::api_ldot<float, 6, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_H_dot_H(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_H_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_H_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_H_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_H_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_H_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_H_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_H_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pH_dot_H(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pH_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_pH_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_pH_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pH_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pH_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_pH_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_pH_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_norm2_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_norm2_H");
  qlab::api_ldot<float, 6, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_norm2_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_norm2_pH");
  qlab::api_ldot<float, 6, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_veqm_H_dot_H(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_H_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_H_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_H_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_H_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_H_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_H_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_H_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pH_dot_H(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pH_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_pH_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_pH_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pH_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pH_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_pH_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_pH_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_norm2_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_norm2_H");
  qlab::api_ldot<float, 6, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_norm2_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_norm2_pH");
  qlab::api_ldot<float, 6, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeq_H_dot_H(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_H_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_H_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_H_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_H_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_H_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_H_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_H_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pH_dot_H(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pH_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_pH_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_pH_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pH_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pH_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_pH_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_pH_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_norm2_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_norm2_H");
  qlab::api_ldot<float, 6, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_norm2_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_norm2_pH");
  qlab::api_ldot<float, 6, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_H_dot_H(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_H_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_H_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_H_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_H_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_H_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_H_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_H_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pH_dot_H(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pH_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_pH_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_pH_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pH_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pH_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_pH_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_pH_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_norm2_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_norm2_H");
  qlab::api_ldot<float, 6, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_norm2_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_norm2_pH");
  qlab::api_ldot<float, 6, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_H_dot_H(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_H_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_H_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_H_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_H_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_H_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_H_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_H_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pH_dot_H(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pH_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_pH_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_pH_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pH_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pH_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_pH_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_pH_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_norm2_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_norm2_H");
  qlab::api_ldot<float, 6, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_norm2_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_norm2_pH");
  qlab::api_ldot<float, 6, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xeqm_H_dot_H(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_H_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_H_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_H_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_H_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_H_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_H_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_H_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pH_dot_H(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pH_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_pH_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_pH_dot_H");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pH_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pH_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_pH_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_pH_dot_pH");
  qlab::api_ldot<float, 6, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_norm2_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_norm2_H");
  qlab::api_ldot<float, 6, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_norm2_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_norm2_pH");
  qlab::api_ldot<float, 6, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veq_D_dot_D(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_D_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_D_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_D_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_D_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_D_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_D_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_D_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pD_dot_D(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pD_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_pD_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_pD_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pD_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pD_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_pD_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_pD_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_norm2_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_veq_norm2_D");
  qlab::api_ldot<float, 12, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_norm2_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_veq_norm2_pD");
  qlab::api_ldot<float, 12, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_D_dot_D(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_D_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_D_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_D_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_D_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_D_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_D_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_D_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pD_dot_D(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pD_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_pD_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_pD_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pD_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pD_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_pD_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_pD_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_norm2_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_norm2_D");
  qlab::api_ldot<float, 12, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_norm2_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_norm2_pD");
  qlab::api_ldot<float, 12, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_D_dot_D(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_D_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_D_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_D_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_D_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_D_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_D_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_D_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pD_dot_D(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pD_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_pD_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_pD_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pD_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pD_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_pD_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_pD_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_norm2_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_norm2_D");
  qlab::api_ldot<float, 12, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_norm2_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_norm2_pD");
  qlab::api_ldot<float, 12, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_veqm_D_dot_D(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_D_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_D_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_D_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_D_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_D_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_D_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_D_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pD_dot_D(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pD_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_pD_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_pD_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pD_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pD_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_pD_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_pD_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_norm2_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_norm2_D");
  qlab::api_ldot<float, 12, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_norm2_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_norm2_pD");
  qlab::api_ldot<float, 12, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeq_D_dot_D(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_D_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_D_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_D_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_D_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_D_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_D_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_D_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pD_dot_D(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pD_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_pD_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_pD_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pD_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pD_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_pD_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_pD_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_norm2_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_norm2_D");
  qlab::api_ldot<float, 12, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_norm2_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_norm2_pD");
  qlab::api_ldot<float, 12, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_D_dot_D(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_D_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_D_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_D_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_D_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_D_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_D_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_D_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pD_dot_D(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pD_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_pD_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_pD_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pD_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pD_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_pD_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_pD_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_norm2_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_norm2_D");
  qlab::api_ldot<float, 12, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_norm2_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_norm2_pD");
  qlab::api_ldot<float, 12, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_D_dot_D(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_D_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_D_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_D_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_D_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_D_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_D_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_D_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pD_dot_D(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pD_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_pD_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_pD_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pD_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pD_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_pD_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_pD_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_norm2_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_norm2_D");
  qlab::api_ldot<float, 12, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_norm2_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_norm2_pD");
  qlab::api_ldot<float, 12, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xeqm_D_dot_D(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_D_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_D_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_D_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_D_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_D_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_D_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_D_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pD_dot_D(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pD_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_pD_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_pD_dot_D");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pD_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pD_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_pD_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_pD_dot_pD");
  qlab::api_ldot<float, 12, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_norm2_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_norm2_D");
  qlab::api_ldot<float, 12, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_norm2_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_norm2_pD");
  qlab::api_ldot<float, 12, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veq_M_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_M_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_M_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_M_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_M_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_M_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_M_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_M_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pM_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pM_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_pM_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_pM_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pM_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pM_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_pM_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_pM_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_M_dot_Ma(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_M_dot_Ma");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_M_dot_pMa(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_M_dot_pMa");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pM_dot_Ma(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pM_dot_Ma");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pM_dot_pMa(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pM_dot_pMa");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_Ma_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_Ma_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_Ma_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_Ma_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pMa_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pMa_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pMa_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pMa_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_norm2_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_veq_norm2_M");
  qlab::api_ldot<float, 9, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_norm2_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_veq_norm2_pM");
  qlab::api_ldot<float, 9, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_M_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_M_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_M_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_M_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_M_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_M_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_M_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_M_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pM_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pM_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_pM_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_pM_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pM_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pM_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_pM_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_pM_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_M_dot_Ma(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_M_dot_Ma");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_M_dot_pMa(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_M_dot_pMa");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pM_dot_Ma(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pM_dot_Ma");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pM_dot_pMa(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pM_dot_pMa");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_Ma_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_Ma_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_Ma_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_Ma_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pMa_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pMa_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pMa_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pMa_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_norm2_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_norm2_M");
  qlab::api_ldot<float, 9, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_norm2_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_norm2_pM");
  qlab::api_ldot<float, 9, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_M_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_M_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_M_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_M_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_M_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_M_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_M_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_M_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pM_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pM_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_pM_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_pM_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pM_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pM_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_pM_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_pM_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_M_dot_Ma(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_M_dot_Ma");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_M_dot_pMa(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_M_dot_pMa");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pM_dot_Ma(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pM_dot_Ma");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pM_dot_pMa(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pM_dot_pMa");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_Ma_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_Ma_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_Ma_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_Ma_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pMa_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pMa_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pMa_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pMa_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_norm2_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_norm2_M");
  qlab::api_ldot<float, 9, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_norm2_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_norm2_pM");
  qlab::api_ldot<float, 9, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_veqm_M_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_M_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_M_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_M_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_M_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_M_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_M_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_M_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pM_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pM_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_pM_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_pM_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pM_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pM_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_pM_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_pM_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_M_dot_Ma(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_M_dot_Ma");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_M_dot_pMa(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_M_dot_pMa");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pM_dot_Ma(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pM_dot_Ma");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pM_dot_pMa(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pM_dot_pMa");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_Ma_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_Ma_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_Ma_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_Ma_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pMa_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pMa_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pMa_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pMa_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_norm2_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_norm2_M");
  qlab::api_ldot<float, 9, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_norm2_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_norm2_pM");
  qlab::api_ldot<float, 9, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeq_M_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_M_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_M_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_M_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_M_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_M_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_M_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_M_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pM_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pM_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_pM_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_pM_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pM_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pM_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_pM_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_pM_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_M_dot_Ma(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_M_dot_Ma");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_M_dot_pMa(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_M_dot_pMa");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pM_dot_Ma(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pM_dot_Ma");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pM_dot_pMa(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pM_dot_pMa");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_Ma_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_Ma_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_Ma_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_Ma_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pMa_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pMa_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pMa_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pMa_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_norm2_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_norm2_M");
  qlab::api_ldot<float, 9, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_norm2_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_norm2_pM");
  qlab::api_ldot<float, 9, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_M_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_M_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_M_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_M_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_M_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_M_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_M_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_M_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pM_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pM_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_pM_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_pM_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pM_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pM_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_pM_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_pM_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_M_dot_Ma(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_M_dot_Ma");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_M_dot_pMa(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_M_dot_pMa");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pM_dot_Ma(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pM_dot_Ma");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pM_dot_pMa(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pM_dot_pMa");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_Ma_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_Ma_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_Ma_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_Ma_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pMa_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pMa_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pMa_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pMa_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_norm2_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_norm2_M");
  qlab::api_ldot<float, 9, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_norm2_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_norm2_pM");
  qlab::api_ldot<float, 9, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_M_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_M_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_M_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_M_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_M_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_M_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_M_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_M_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pM_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pM_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_pM_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_pM_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pM_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pM_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_pM_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_pM_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_M_dot_Ma(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_M_dot_Ma");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_M_dot_pMa(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_M_dot_pMa");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pM_dot_Ma(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pM_dot_Ma");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pM_dot_pMa(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pM_dot_pMa");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_Ma_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_Ma_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_Ma_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_Ma_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pMa_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pMa_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pMa_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pMa_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_norm2_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_norm2_M");
  qlab::api_ldot<float, 9, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_norm2_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_norm2_pM");
  qlab::api_ldot<float, 9, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xeqm_M_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_M_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_M_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_M_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_M_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_M_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_M_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_M_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pM_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pM_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_pM_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_pM_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pM_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pM_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_pM_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_pM_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_M_dot_Ma(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_M_dot_Ma");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_M_dot_pMa(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_M_dot_pMa");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pM_dot_Ma(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pM_dot_Ma");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pM_dot_pMa(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pM_dot_pMa");
  qlab::api_ldot<float, 9, qlab::LD_DOT_AA, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_Ma_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_Ma_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_Ma_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_Ma_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pMa_dot_M(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pMa_dot_M");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pMa_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pMa_dot_pM");
  qlab::api_ldot<float, 9, qlab::LD_ADOT, qlab::PERM_M>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_norm2_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_norm2_M");
  qlab::api_ldot<float, 9, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_norm2_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_norm2_pM");
  qlab::api_ldot<float, 9, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veq_P_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_P_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_P_dot_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_P_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_P_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_P_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_P_dot_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_P_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pP_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pP_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_pP_dot_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_pP_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pP_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pP_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_re_pP_dot_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veq_re_pP_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_P_dot_Pa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_P_dot_Pa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_P_dot_pPa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_P_dot_pPa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pP_dot_Pa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pP_dot_Pa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pP_dot_pPa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pP_dot_pPa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_Pa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_Pa_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_Pa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_Pa_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pPa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pPa_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_veq_pPa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veq_pPa_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_norm2_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_veq_norm2_P");
  qlab::api_ldot<float, 144, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_veq_norm2_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_veq_norm2_pP");
  qlab::api_ldot<float, 144, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_P_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_P_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_P_dot_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_P_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_P_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_P_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_P_dot_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_P_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pP_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pP_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_pP_dot_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_pP_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pP_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pP_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_re_pP_dot_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_re_pP_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_P_dot_Pa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_P_dot_Pa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_P_dot_pPa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_P_dot_pPa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pP_dot_Pa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pP_dot_Pa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pP_dot_pPa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pP_dot_pPa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_Pa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_Pa_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_Pa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_Pa_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pPa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pPa_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vpeq_pPa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vpeq_pPa_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_norm2_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_norm2_P");
  qlab::api_ldot<float, 144, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_vpeq_norm2_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_vpeq_norm2_pP");
  qlab::api_ldot<float, 144, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_P_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_P_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_P_dot_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_P_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_P_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_P_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_P_dot_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_P_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pP_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pP_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_pP_dot_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_pP_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pP_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pP_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_re_pP_dot_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_re_pP_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_P_dot_Pa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_P_dot_Pa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_P_dot_pPa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_P_dot_pPa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pP_dot_Pa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pP_dot_Pa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pP_dot_pPa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pP_dot_pPa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_Pa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_Pa_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_Pa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_Pa_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pPa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pPa_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_vmeq_pPa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_vmeq_pPa_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_norm2_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_norm2_P");
  qlab::api_ldot<float, 144, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_vmeq_norm2_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_vmeq_norm2_pP");
  qlab::api_ldot<float, 144, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_veqm_P_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_P_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_P_dot_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_P_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_P_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_P_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_P_dot_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_P_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pP_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pP_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_pP_dot_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_pP_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pP_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pP_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_re_pP_dot_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_re_pP_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_P_dot_Pa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_P_dot_Pa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_P_dot_pPa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_P_dot_pPa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pP_dot_Pa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pP_dot_Pa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pP_dot_pPa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pP_dot_pPa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_Pa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_Pa_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_Pa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_Pa_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pPa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pPa_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_veqm_pPa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_C_veqm_pPa_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_norm2_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_norm2_P");
  qlab::api_ldot<float, 144, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_veqm_norm2_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_R_veqm_norm2_pP");
  qlab::api_ldot<float, 144, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeq_P_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_P_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_P_dot_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_P_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_P_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_P_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_P_dot_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_P_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pP_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pP_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_pP_dot_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_pP_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pP_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pP_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_re_pP_dot_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_re_pP_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_P_dot_Pa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_P_dot_Pa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_P_dot_pPa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_P_dot_pPa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pP_dot_Pa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pP_dot_Pa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pP_dot_pPa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pP_dot_pPa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_Pa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_Pa_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_Pa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_Pa_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pPa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pPa_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xeq_pPa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeq_pPa_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_norm2_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_norm2_P");
  qlab::api_ldot<float, 144, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_R_xeq_norm2_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeq_norm2_pP");
  qlab::api_ldot<float, 144, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_P_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_P_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_P_dot_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_P_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_P_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_P_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_P_dot_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_P_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pP_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pP_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_pP_dot_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_pP_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pP_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pP_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_re_pP_dot_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_re_pP_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_P_dot_Pa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_P_dot_Pa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_P_dot_pPa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_P_dot_pPa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pP_dot_Pa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pP_dot_Pa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pP_dot_pPa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pP_dot_pPa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_Pa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_Pa_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_Pa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_Pa_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pPa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pPa_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xpeq_pPa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xpeq_pPa_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_norm2_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_norm2_P");
  qlab::api_ldot<float, 144, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_R_xpeq_norm2_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xpeq_norm2_pP");
  qlab::api_ldot<float, 144, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_P_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_P_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_P_dot_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_P_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_P_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_P_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_P_dot_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_P_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pP_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pP_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_pP_dot_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_pP_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pP_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pP_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_re_pP_dot_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_re_pP_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_P_dot_Pa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_P_dot_Pa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_P_dot_pPa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_P_dot_pPa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pP_dot_Pa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pP_dot_Pa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pP_dot_pPa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pP_dot_pPa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_Pa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_Pa_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_Pa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_Pa_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pPa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pPa_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xmeq_pPa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xmeq_pPa_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_norm2_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_norm2_P");
  qlab::api_ldot<float, 144, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_R_xmeq_norm2_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xmeq_norm2_pP");
  qlab::api_ldot<float, 144, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_C_xeqm_P_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_P_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_P_dot_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_P_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_P_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_P_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_P_dot_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_P_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pP_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pP_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_pP_dot_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_pP_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pP_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pP_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_DOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_re_pP_dot_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_re_pP_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_REDOT, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_P_dot_Pa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_P_dot_Pa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_P_dot_pPa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_P_dot_pPa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pP_dot_Pa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pP_dot_Pa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pP_dot_pPa(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pP_dot_pPa");
  qlab::api_ldot<float, 144, qlab::LD_DOT_AA, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_Pa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_Pa_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_Pa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_Pa_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pPa_dot_P(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pPa_dot_P");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_C_xeqm_pPa_dot_pP(QLA_F_Complex *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, QLA_F3_DiracPropagator *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_C_xeqm_pPa_dot_pP");
  qlab::api_ldot<float, 144, qlab::LD_ADOT, qlab::PERM_P>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_norm2_P(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_norm2_P");
  qlab::api_ldot<float, 144, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_R_xeqm_norm2_pP(QLA_F_Real *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_R_xeqm_norm2_pP");
  qlab::api_ldot<float, 144, qlab::LD_NORM2, qlab::PERM_ID>("F3_ldot", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_M_veq_V_times_Va(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_M_veq_V_times_Va");
  qlab::api_outer<float>("F3_outer", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_M_veq_V_times_pVa(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_M_veq_V_times_pVa");
  qlab::api_outer<float>("F3_outer", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_M_veq_pV_times_Va(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_M_veq_pV_times_Va");
  qlab::api_outer<float>("F3_outer", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_M_veq_pV_times_pVa(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_M_veq_pV_times_pVa");
  qlab::api_outer<float>("F3_outer", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_M_vpeq_V_times_Va(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_M_vpeq_V_times_Va");
  qlab::api_outer<float>("F3_outer", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_M_vpeq_V_times_pVa(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_M_vpeq_V_times_pVa");
  qlab::api_outer<float>("F3_outer", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_M_vpeq_pV_times_Va(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_M_vpeq_pV_times_Va");
  qlab::api_outer<float>("F3_outer", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_M_vpeq_pV_times_pVa(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_M_vpeq_pV_times_pVa");
  qlab::api_outer<float>("F3_outer", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_M_vmeq_V_times_Va(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_M_vmeq_V_times_Va");
  qlab::api_outer<float>("F3_outer", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_M_vmeq_V_times_pVa(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_M_vmeq_V_times_pVa");
  qlab::api_outer<float>("F3_outer", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_M_vmeq_pV_times_Va(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_M_vmeq_pV_times_Va");
  qlab::api_outer<float>("F3_outer", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_M_vmeq_pV_times_pVa(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_M_vmeq_pV_times_pVa");
  qlab::api_outer<float>("F3_outer", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_M_veqm_V_times_Va(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_M_veqm_V_times_Va");
  qlab::api_outer<float>("F3_outer", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_M_veqm_V_times_pVa(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_M_veqm_V_times_pVa");
  qlab::api_outer<float>("F3_outer", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_M_veqm_pV_times_Va(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_M_veqm_pV_times_Va");
  qlab::api_outer<float>("F3_outer", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_M_veqm_pV_times_pVa(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_M_veqm_pV_times_pVa");
  qlab::api_outer<float>("F3_outer", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_M_xeq_V_times_Va(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xeq_V_times_Va");
  qlab::api_outer<float>("F3_outer", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_M_xeq_V_times_pVa(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xeq_V_times_pVa");
  qlab::api_outer<float>("F3_outer", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_M_xeq_pV_times_Va(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xeq_pV_times_Va");
  qlab::api_outer<float>("F3_outer", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_M_xeq_pV_times_pVa(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xeq_pV_times_pVa");
  qlab::api_outer<float>("F3_outer", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F3_M_xpeq_V_times_Va(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xpeq_V_times_Va");
  qlab::api_outer<float>("F3_outer", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_M_xpeq_V_times_pVa(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xpeq_V_times_pVa");
  qlab::api_outer<float>("F3_outer", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_M_xpeq_pV_times_Va(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xpeq_pV_times_Va");
  qlab::api_outer<float>("F3_outer", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_M_xpeq_pV_times_pVa(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xpeq_pV_times_pVa");
  qlab::api_outer<float>("F3_outer", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F3_M_xmeq_V_times_Va(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xmeq_V_times_Va");
  qlab::api_outer<float>("F3_outer", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_M_xmeq_V_times_pVa(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xmeq_V_times_pVa");
  qlab::api_outer<float>("F3_outer", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_M_xmeq_pV_times_Va(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xmeq_pV_times_Va");
  qlab::api_outer<float>("F3_outer", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_M_xmeq_pV_times_pVa(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xmeq_pV_times_pVa");
  qlab::api_outer<float>("F3_outer", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F3_M_xeqm_V_times_Va(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xeqm_V_times_Va");
  qlab::api_outer<float>("F3_outer", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_M_xeqm_V_times_pVa(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xeqm_V_times_pVa");
  qlab::api_outer<float>("F3_outer", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_M_xeqm_pV_times_Va(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xeqm_pV_times_Va");
  qlab::api_outer<float>("F3_outer", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F3_M_xeqm_pV_times_pVa(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_M_xeqm_pV_times_pVa");
  qlab::api_outer<float>("F3_outer", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

}  // extern "C"
