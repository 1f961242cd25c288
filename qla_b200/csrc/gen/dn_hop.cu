// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA DN hop entry points (extern "C"), reference: lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_DN_H_veq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veq_spproj_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veq_spproj_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_spproj_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_spproj_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_sprecon_M_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_sprecon_M_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_sprecon_M_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_sprecon_M_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_sprecon_M_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_sprecon_M_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veq_spproj_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veq_spproj_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_spproj_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_spproj_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_sprecon_Ma_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_sprecon_Ma_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_sprecon_Ma_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_sprecon_Ma_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_sprecon_Ma_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_sprecon_Ma_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veq_spproj_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veq_spproj_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_spproj_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_spproj_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_sprecon_pM_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_sprecon_pM_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_sprecon_pM_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_sprecon_pM_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_sprecon_pM_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_sprecon_pM_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veq_spproj_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veq_spproj_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_spproj_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_spproj_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_sprecon_pMa_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_sprecon_pMa_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_sprecon_pMa_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_sprecon_pMa_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_sprecon_pMa_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_sprecon_pMa_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_spproj_D(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_spproj_D");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojDOp<double, 2>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojDOp<double, 3>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojDOp<double, 4>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojDOp<double, 8>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_spproj_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojDOp<double, 2>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojDOp<double, 3>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojDOp<double, 4>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojDOp<double, 8>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_spproj_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vpeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vpeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vpeq_spproj_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vpeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vpeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vpeq_spproj_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_spproj_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_spproj_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_sprecon_M_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_sprecon_M_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_sprecon_M_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_sprecon_M_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_sprecon_M_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_sprecon_M_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vpeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vpeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vpeq_spproj_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vpeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vpeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vpeq_spproj_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_spproj_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_spproj_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_sprecon_Ma_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_sprecon_Ma_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_sprecon_Ma_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_sprecon_Ma_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_sprecon_Ma_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_sprecon_Ma_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vpeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vpeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vpeq_spproj_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vpeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vpeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vpeq_spproj_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_spproj_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_spproj_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_sprecon_pM_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_sprecon_pM_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_sprecon_pM_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_sprecon_pM_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_sprecon_pM_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_sprecon_pM_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vpeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vpeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vpeq_spproj_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vpeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vpeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vpeq_spproj_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_spproj_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_spproj_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_sprecon_pMa_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_sprecon_pMa_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_sprecon_pMa_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_sprecon_pMa_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_sprecon_pMa_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_sprecon_pMa_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_spproj_D");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojDOp<double, 2>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojDOp<double, 3>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojDOp<double, 4>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojDOp<double, 8>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_spproj_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojDOp<double, 2>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojDOp<double, 3>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojDOp<double, 4>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojDOp<double, 8>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_spproj_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vmeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vmeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vmeq_spproj_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vmeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vmeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vmeq_spproj_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_spproj_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_spproj_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_sprecon_M_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_sprecon_M_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_sprecon_M_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_sprecon_M_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_sprecon_M_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_sprecon_M_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vmeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vmeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vmeq_spproj_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vmeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vmeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vmeq_spproj_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_spproj_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_spproj_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_sprecon_Ma_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_sprecon_Ma_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_sprecon_Ma_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_sprecon_Ma_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_sprecon_Ma_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_sprecon_Ma_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vmeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vmeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vmeq_spproj_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vmeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vmeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vmeq_spproj_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_spproj_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_spproj_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_sprecon_pM_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_sprecon_pM_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_sprecon_pM_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_sprecon_pM_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_sprecon_pM_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_sprecon_pM_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vmeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vmeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vmeq_spproj_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vmeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vmeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vmeq_spproj_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_spproj_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_spproj_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_sprecon_pMa_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_sprecon_pMa_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_sprecon_pMa_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_sprecon_pMa_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_sprecon_pMa_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_sprecon_pMa_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_spproj_D");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojDOp<double, 2>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojDOp<double, 3>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojDOp<double, 4>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojDOp<double, 8>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_spproj_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojDOp<double, 2>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojDOp<double, 3>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojDOp<double, 4>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojDOp<double, 8>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_spproj_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veqm_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veqm_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veqm_spproj_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veqm_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veqm_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veqm_spproj_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_spproj_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_spproj_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_sprecon_M_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_sprecon_M_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_sprecon_M_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_sprecon_M_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_sprecon_M_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_sprecon_M_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veqm_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veqm_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veqm_spproj_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veqm_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veqm_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veqm_spproj_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_spproj_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_spproj_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_sprecon_Ma_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_sprecon_Ma_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_sprecon_Ma_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_sprecon_Ma_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_sprecon_Ma_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_sprecon_Ma_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veqm_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veqm_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veqm_spproj_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veqm_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veqm_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veqm_spproj_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_spproj_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_spproj_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_sprecon_pM_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_sprecon_pM_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_sprecon_pM_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_sprecon_pM_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_sprecon_pM_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_sprecon_pM_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veqm_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veqm_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veqm_spproj_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veqm_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veqm_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veqm_spproj_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_spproj_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_spproj_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_sprecon_pMa_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_sprecon_pMa_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_sprecon_pMa_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_sprecon_pMa_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_sprecon_pMa_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_sprecon_pMa_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_spproj_D(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_spproj_D");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojDOp<double, 2>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojDOp<double, 3>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojDOp<double, 4>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojDOp<double, 8>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_spproj_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_spproj_pD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojDOp<double, 2>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojDOp<double, 3>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojDOp<double, 4>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojDOp<double, 8>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_spproj_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeq_spproj_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeq_spproj_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_spproj_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_spproj_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_sprecon_M_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_sprecon_M_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_sprecon_M_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_sprecon_M_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_sprecon_M_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_sprecon_M_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeq_spproj_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeq_spproj_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_spproj_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_spproj_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_sprecon_Ma_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_sprecon_Ma_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_sprecon_Ma_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_sprecon_Ma_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_sprecon_Ma_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_sprecon_Ma_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeq_spproj_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeq_spproj_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_spproj_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_spproj_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_sprecon_pM_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_sprecon_pM_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_sprecon_pM_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_sprecon_pM_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_sprecon_pM_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_sprecon_pM_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeq_spproj_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeq_spproj_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_spproj_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_spproj_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_sprecon_pMa_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_sprecon_pMa_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_sprecon_pMa_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_sprecon_pMa_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_sprecon_pMa_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_sprecon_pMa_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_spproj_D");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojDOp<double, 2>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojDOp<double, 3>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojDOp<double, 4>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojDOp<double, 8>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_spproj_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojDOp<double, 2>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojDOp<double, 3>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojDOp<double, 4>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojDOp<double, 8>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_spproj_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xpeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xpeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xpeq_spproj_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xpeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xpeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xpeq_spproj_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_spproj_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_spproj_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_sprecon_M_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_sprecon_M_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_sprecon_M_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_sprecon_M_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_sprecon_M_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_sprecon_M_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xpeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xpeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xpeq_spproj_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xpeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xpeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xpeq_spproj_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_spproj_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_spproj_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_sprecon_Ma_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_sprecon_Ma_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_sprecon_Ma_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_sprecon_Ma_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_sprecon_Ma_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_sprecon_Ma_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xpeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xpeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xpeq_spproj_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xpeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xpeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xpeq_spproj_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_spproj_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_spproj_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_sprecon_pM_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_sprecon_pM_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_sprecon_pM_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_sprecon_pM_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_sprecon_pM_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_sprecon_pM_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xpeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xpeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xpeq_spproj_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xpeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xpeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xpeq_spproj_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_spproj_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_spproj_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_sprecon_pMa_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_sprecon_pMa_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_sprecon_pMa_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_sprecon_pMa_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_sprecon_pMa_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_sprecon_pMa_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_spproj_D");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojDOp<double, 2>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojDOp<double, 3>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojDOp<double, 4>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojDOp<double, 8>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_spproj_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojDOp<double, 2>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojDOp<double, 3>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojDOp<double, 4>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojDOp<double, 8>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_spproj_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xmeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xmeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xmeq_spproj_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xmeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xmeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xmeq_spproj_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_spproj_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_spproj_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_sprecon_M_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_sprecon_M_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_sprecon_M_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_sprecon_M_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_sprecon_M_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_sprecon_M_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xmeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xmeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xmeq_spproj_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xmeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xmeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xmeq_spproj_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_spproj_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_spproj_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_sprecon_Ma_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_sprecon_Ma_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_sprecon_Ma_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_sprecon_Ma_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_sprecon_Ma_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_sprecon_Ma_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xmeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xmeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xmeq_spproj_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xmeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xmeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xmeq_spproj_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_spproj_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_spproj_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_sprecon_pM_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_sprecon_pM_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_sprecon_pM_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_sprecon_pM_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_sprecon_pM_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_sprecon_pM_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xmeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xmeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xmeq_spproj_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xmeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xmeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xmeq_spproj_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_spproj_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_spproj_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_sprecon_pMa_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_sprecon_pMa_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_sprecon_pMa_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_sprecon_pMa_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_sprecon_pMa_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_sprecon_pMa_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_spproj_D");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojDOp<double, 2>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojDOp<double, 3>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojDOp<double, 4>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojDOp<double, 8>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_spproj_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojDOp<double, 2>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojDOp<double, 3>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojDOp<double, 4>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojDOp<double, 8>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_spproj_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeqm_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeqm_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeqm_spproj_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeqm_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeqm_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeqm_spproj_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_spproj_M_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_spproj_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_spproj_M_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_spproj_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_sprecon_M_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_sprecon_M_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_sprecon_M_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_sprecon_M_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_sprecon_M_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_sprecon_M_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeqm_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeqm_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeqm_spproj_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeqm_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeqm_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeqm_spproj_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_spproj_Ma_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_spproj_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_spproj_Ma_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_spproj_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_sprecon_Ma_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_sprecon_Ma_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_sprecon_Ma_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_sprecon_Ma_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_sprecon_Ma_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_sprecon_Ma_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeqm_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeqm_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeqm_spproj_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeqm_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeqm_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeqm_spproj_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_spproj_pM_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_spproj_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_spproj_pM_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_spproj_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_sprecon_pM_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_sprecon_pM_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_sprecon_pM_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_sprecon_pM_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_sprecon_pM_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_sprecon_pM_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeqm_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeqm_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeqm_spproj_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeqm_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeqm_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeqm_spproj_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_spproj_pMa_times_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_spproj_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_spproj_pMa_times_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_spproj_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_sprecon_pMa_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_sprecon_pMa_times_H");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_sprecon_pMa_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_sprecon_pMa_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_sprecon_pMa_times_pH");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_sprecon_pMa_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_spproj_D");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojDOp<double, 2>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojDOp<double, 3>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojDOp<double, 4>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojDOp<double, 8>>("DN_hop_Dspproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_spproj_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_spproj_pD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojDOp<double, 2>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojDOp<double, 3>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojDOp<double, 4>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojDOp<double, 8>>("DN_hop_Dspproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_spproj_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_eq_spproj_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_eq_spproj_M_times_xD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_eq_spproj_M_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_eq_spproj_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_eq_spproj_M_times_xD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_eq_spproj_M_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_eq_sprecon_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_eq_sprecon_M_times_xH");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_eq_sprecon_M_times_xH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_eq_spproj_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_eq_spproj_Ma_times_xD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_eq_spproj_Ma_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_eq_spproj_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_eq_spproj_Ma_times_xD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_eq_spproj_Ma_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_eq_sprecon_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_eq_sprecon_Ma_times_xH");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_eq_sprecon_Ma_times_xH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_peq_spproj_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_peq_spproj_M_times_xD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_peq_spproj_M_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_peq_spproj_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_peq_spproj_M_times_xD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_peq_spproj_M_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_peq_sprecon_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_peq_sprecon_M_times_xH");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_peq_sprecon_M_times_xH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_peq_spproj_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_peq_spproj_Ma_times_xD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_peq_spproj_Ma_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_peq_spproj_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_peq_spproj_Ma_times_xD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_peq_spproj_Ma_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_peq_sprecon_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_peq_sprecon_Ma_times_xH");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_peq_sprecon_Ma_times_xH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_meq_spproj_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_meq_spproj_M_times_xD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_meq_spproj_M_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_meq_spproj_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_meq_spproj_M_times_xD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_meq_spproj_M_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_meq_sprecon_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_meq_sprecon_M_times_xH");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_meq_sprecon_M_times_xH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_meq_spproj_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_meq_spproj_Ma_times_xD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_meq_spproj_Ma_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_meq_spproj_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_meq_spproj_Ma_times_xD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_meq_spproj_Ma_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_meq_sprecon_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_meq_sprecon_Ma_times_xH");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_meq_sprecon_Ma_times_xH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_eqm_spproj_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_eqm_spproj_M_times_xD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 2>>("DN_hop_Hspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_eqm_spproj_M_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_eqm_spproj_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_eqm_spproj_M_times_xD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, false, 4>>("DN_hop_Dspprojfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_eqm_spproj_M_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_eqm_sprecon_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_eqm_sprecon_M_times_xH");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, false>>("DN_hop_Dspreconfalse", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_eqm_sprecon_M_times_xH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_eqm_spproj_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_eqm_spproj_Ma_times_xD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 2>>("DN_hop_Hspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_eqm_spproj_Ma_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_eqm_spproj_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_eqm_spproj_Ma_times_xD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojMultOp<double, 2, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojMultOp<double, 3, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojMultOp<double, 4, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojMultOp<double, 8, true, 4>>("DN_hop_Dspprojtrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_eqm_spproj_Ma_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_eqm_sprecon_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_eqm_sprecon_Ma_times_xH");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconMultOp<double, 2, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconMultOp<double, 3, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconMultOp<double, 4, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconMultOp<double, 8, true>>("DN_hop_Dsprecontrue", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_eqm_sprecon_Ma_times_xH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

}  // extern "C"
