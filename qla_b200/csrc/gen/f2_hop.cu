// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F2 hop entry points (extern "C"), reference: lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_F2_H_veq_spproj_M_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_veq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_veq_spproj_M_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_veq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_spproj_M_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_spproj_M_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_sprecon_M_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_sprecon_M_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_sprecon_M_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_sprecon_M_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_veq_spproj_Ma_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_veq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_veq_spproj_Ma_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_veq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_spproj_Ma_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_spproj_Ma_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_sprecon_Ma_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_sprecon_Ma_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_sprecon_Ma_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_sprecon_Ma_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_veq_spproj_pM_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_veq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_veq_spproj_pM_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_veq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_spproj_pM_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_spproj_pM_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_sprecon_pM_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_sprecon_pM_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_sprecon_pM_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_sprecon_pM_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_veq_spproj_pMa_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_veq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_veq_spproj_pMa_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_veq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_spproj_pMa_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_spproj_pMa_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_sprecon_pMa_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_sprecon_pMa_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_sprecon_pMa_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_sprecon_pMa_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_spproj_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_spproj_D");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojDOp<float, 2>>("F2_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veq_spproj_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojDOp<float, 2>>("F2_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_vpeq_spproj_M_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_vpeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_vpeq_spproj_M_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_vpeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_spproj_M_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_spproj_M_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_sprecon_M_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_sprecon_M_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_sprecon_M_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_sprecon_M_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_vpeq_spproj_Ma_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_vpeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_vpeq_spproj_Ma_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_vpeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_spproj_Ma_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_spproj_Ma_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_sprecon_Ma_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_sprecon_Ma_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_sprecon_Ma_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_sprecon_Ma_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_vpeq_spproj_pM_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_vpeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_vpeq_spproj_pM_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_vpeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_spproj_pM_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_spproj_pM_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_sprecon_pM_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_sprecon_pM_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_sprecon_pM_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_sprecon_pM_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_vpeq_spproj_pMa_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_vpeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_vpeq_spproj_pMa_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_vpeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_spproj_pMa_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_spproj_pMa_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_sprecon_pMa_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_sprecon_pMa_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_sprecon_pMa_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_sprecon_pMa_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_spproj_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_spproj_D");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojDOp<float, 2>>("F2_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vpeq_spproj_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojDOp<float, 2>>("F2_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_vmeq_spproj_M_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_vmeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_vmeq_spproj_M_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_vmeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_spproj_M_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_spproj_M_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_sprecon_M_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_sprecon_M_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_sprecon_M_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_sprecon_M_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_vmeq_spproj_Ma_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_vmeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_vmeq_spproj_Ma_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_vmeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_spproj_Ma_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_spproj_Ma_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_sprecon_Ma_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_sprecon_Ma_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_sprecon_Ma_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_sprecon_Ma_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_vmeq_spproj_pM_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_vmeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_vmeq_spproj_pM_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_vmeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_spproj_pM_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_spproj_pM_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_sprecon_pM_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_sprecon_pM_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_sprecon_pM_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_sprecon_pM_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_vmeq_spproj_pMa_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_vmeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_vmeq_spproj_pMa_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_vmeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_spproj_pMa_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_spproj_pMa_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_sprecon_pMa_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_sprecon_pMa_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_sprecon_pMa_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_sprecon_pMa_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_spproj_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_spproj_D");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojDOp<float, 2>>("F2_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_vmeq_spproj_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojDOp<float, 2>>("F2_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_veqm_spproj_M_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_veqm_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_veqm_spproj_M_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_veqm_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_spproj_M_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_spproj_M_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_sprecon_M_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_sprecon_M_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_sprecon_M_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_sprecon_M_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_veqm_spproj_Ma_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_veqm_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_veqm_spproj_Ma_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_veqm_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_spproj_Ma_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_spproj_Ma_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_sprecon_Ma_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_sprecon_Ma_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_sprecon_Ma_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_sprecon_Ma_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_veqm_spproj_pM_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_veqm_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_veqm_spproj_pM_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_veqm_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_spproj_pM_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_spproj_pM_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_sprecon_pM_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_sprecon_pM_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_sprecon_pM_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_sprecon_pM_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_veqm_spproj_pMa_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_veqm_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_veqm_spproj_pMa_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_veqm_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_spproj_pMa_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_spproj_pMa_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_sprecon_pMa_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_sprecon_pMa_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_sprecon_pMa_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_sprecon_pMa_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_spproj_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_spproj_D");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojDOp<float, 2>>("F2_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_veqm_spproj_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_spproj_pD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojDOp<float, 2>>("F2_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xeq_spproj_M_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xeq_spproj_M_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_spproj_M_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_spproj_M_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_sprecon_M_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_sprecon_M_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_sprecon_M_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_sprecon_M_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xeq_spproj_Ma_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xeq_spproj_Ma_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_spproj_Ma_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_spproj_Ma_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_sprecon_Ma_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_sprecon_Ma_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_sprecon_Ma_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_sprecon_Ma_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xeq_spproj_pM_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xeq_spproj_pM_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_spproj_pM_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_spproj_pM_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_sprecon_pM_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_sprecon_pM_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_sprecon_pM_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_sprecon_pM_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xeq_spproj_pMa_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xeq_spproj_pMa_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_spproj_pMa_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_spproj_pMa_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_sprecon_pMa_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_sprecon_pMa_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_sprecon_pMa_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_sprecon_pMa_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_spproj_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_spproj_D");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojDOp<float, 2>>("F2_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeq_spproj_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojDOp<float, 2>>("F2_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xpeq_spproj_M_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xpeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xpeq_spproj_M_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xpeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_spproj_M_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_spproj_M_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_sprecon_M_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_sprecon_M_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_sprecon_M_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_sprecon_M_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xpeq_spproj_Ma_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xpeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xpeq_spproj_Ma_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xpeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_spproj_Ma_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_spproj_Ma_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_sprecon_Ma_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_sprecon_Ma_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_sprecon_Ma_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_sprecon_Ma_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xpeq_spproj_pM_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xpeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xpeq_spproj_pM_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xpeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_spproj_pM_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_spproj_pM_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_sprecon_pM_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_sprecon_pM_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_sprecon_pM_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_sprecon_pM_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xpeq_spproj_pMa_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xpeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xpeq_spproj_pMa_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xpeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_spproj_pMa_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_spproj_pMa_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_sprecon_pMa_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_sprecon_pMa_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_sprecon_pMa_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_sprecon_pMa_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_spproj_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_spproj_D");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojDOp<float, 2>>("F2_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xpeq_spproj_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojDOp<float, 2>>("F2_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xmeq_spproj_M_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xmeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xmeq_spproj_M_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xmeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_spproj_M_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_spproj_M_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_sprecon_M_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_sprecon_M_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_sprecon_M_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_sprecon_M_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xmeq_spproj_Ma_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xmeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xmeq_spproj_Ma_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xmeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_spproj_Ma_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_spproj_Ma_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_sprecon_Ma_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_sprecon_Ma_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_sprecon_Ma_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_sprecon_Ma_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xmeq_spproj_pM_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xmeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xmeq_spproj_pM_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xmeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_spproj_pM_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_spproj_pM_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_sprecon_pM_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_sprecon_pM_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_sprecon_pM_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_sprecon_pM_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xmeq_spproj_pMa_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xmeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xmeq_spproj_pMa_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xmeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_spproj_pMa_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_spproj_pMa_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_sprecon_pMa_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_sprecon_pMa_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_sprecon_pMa_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_sprecon_pMa_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_spproj_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_spproj_D");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojDOp<float, 2>>("F2_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xmeq_spproj_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojDOp<float, 2>>("F2_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xeqm_spproj_M_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeqm_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xeqm_spproj_M_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeqm_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_spproj_M_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_spproj_M_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_sprecon_M_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_sprecon_M_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_sprecon_M_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_sprecon_M_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xeqm_spproj_Ma_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeqm_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xeqm_spproj_Ma_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeqm_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_spproj_Ma_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_spproj_Ma_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_sprecon_Ma_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_sprecon_Ma_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_sprecon_Ma_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_sprecon_Ma_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xeqm_spproj_pM_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeqm_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xeqm_spproj_pM_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeqm_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_spproj_pM_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_spproj_pM_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_sprecon_pM_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_sprecon_pM_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_sprecon_pM_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_sprecon_pM_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xeqm_spproj_pMa_times_D(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeqm_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_xeqm_spproj_pMa_times_pD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeqm_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_spproj_pMa_times_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_spproj_pMa_times_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_sprecon_pMa_times_H(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_sprecon_pMa_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_sprecon_pMa_times_pH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_sprecon_pMa_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_spproj_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_spproj_D");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojDOp<float, 2>>("F2_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_xeqm_spproj_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_spproj_pD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojDOp<float, 2>>("F2_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_eq_spproj_M_times_xD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_eq_spproj_M_times_xD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_eq_spproj_M_times_xD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_eq_spproj_M_times_xD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_eq_sprecon_M_times_xH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_eq_sprecon_M_times_xH");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_eq_spproj_Ma_times_xD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_eq_spproj_Ma_times_xD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_eq_spproj_Ma_times_xD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_eq_spproj_Ma_times_xD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_eq_sprecon_Ma_times_xH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_eq_sprecon_Ma_times_xH");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_peq_spproj_M_times_xD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_peq_spproj_M_times_xD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_peq_spproj_M_times_xD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_peq_spproj_M_times_xD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_peq_sprecon_M_times_xH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_peq_sprecon_M_times_xH");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_peq_spproj_Ma_times_xD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_peq_spproj_Ma_times_xD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_peq_spproj_Ma_times_xD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_peq_spproj_Ma_times_xD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_peq_sprecon_Ma_times_xH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_peq_sprecon_Ma_times_xH");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_meq_spproj_M_times_xD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_meq_spproj_M_times_xD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_meq_spproj_M_times_xD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_meq_spproj_M_times_xD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_meq_sprecon_M_times_xH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_meq_sprecon_M_times_xH");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_meq_spproj_Ma_times_xD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_meq_spproj_Ma_times_xD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_meq_spproj_Ma_times_xD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_meq_spproj_Ma_times_xD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_meq_sprecon_Ma_times_xH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_meq_sprecon_Ma_times_xH");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_eqm_spproj_M_times_xD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_eqm_spproj_M_times_xD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 2>>("F2_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_eqm_spproj_M_times_xD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_eqm_spproj_M_times_xD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojMultOp<float, 2, false, 4>>("F2_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_eqm_sprecon_M_times_xH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_eqm_sprecon_M_times_xH");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconMultOp<float, 2, false>>("F2_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_H_eqm_spproj_Ma_times_xD(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_H_eqm_spproj_Ma_times_xD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 2>>("F2_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_eqm_spproj_Ma_times_xD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_eqm_spproj_Ma_times_xD");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpprojMultOp<float, 2, true, 4>>("F2_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F2_D_eqm_sprecon_Ma_times_xH(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F2_D_eqm_sprecon_Ma_times_xH");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconMultOp<float, 2, true>>("F2_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign);
}

}  // extern "C"
