// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA DN spproj entry points (extern "C"), reference: lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_DN_H_veq_spproj_D(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veq_spproj_D");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojOp<double, 2>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojOp<double, 3>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojOp<double, 4>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojOp<double, 8>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veq_spproj_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojOp<double, 2>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojOp<double, 3>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojOp<double, 4>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojOp<double, 8>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veq_spproj_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vpeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vpeq_spproj_D");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojOp<double, 2>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojOp<double, 3>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojOp<double, 4>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojOp<double, 8>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vpeq_spproj_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vpeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vpeq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojOp<double, 2>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojOp<double, 3>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojOp<double, 4>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojOp<double, 8>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vpeq_spproj_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vmeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vmeq_spproj_D");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojOp<double, 2>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojOp<double, 3>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojOp<double, 4>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojOp<double, 8>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vmeq_spproj_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vmeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_vmeq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojOp<double, 2>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojOp<double, 3>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojOp<double, 4>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojOp<double, 8>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vmeq_spproj_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veqm_spproj_D(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veqm_spproj_D");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojOp<double, 2>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojOp<double, 3>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojOp<double, 4>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojOp<double, 8>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veqm_spproj_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veqm_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_H_veqm_spproj_pD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojOp<double, 2>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojOp<double, 3>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojOp<double, 4>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojOp<double, 8>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veqm_spproj_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeq_spproj_D");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojOp<double, 2>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojOp<double, 3>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojOp<double, 4>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojOp<double, 8>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeq_spproj_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojOp<double, 2>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojOp<double, 3>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojOp<double, 4>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojOp<double, 8>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeq_spproj_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xpeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xpeq_spproj_D");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojOp<double, 2>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojOp<double, 3>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojOp<double, 4>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojOp<double, 8>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xpeq_spproj_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xpeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xpeq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojOp<double, 2>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojOp<double, 3>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojOp<double, 4>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojOp<double, 8>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xpeq_spproj_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xmeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xmeq_spproj_D");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojOp<double, 2>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojOp<double, 3>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojOp<double, 4>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojOp<double, 8>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xmeq_spproj_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xmeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xmeq_spproj_pD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojOp<double, 2>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojOp<double, 3>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojOp<double, 4>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojOp<double, 8>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xmeq_spproj_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeqm_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeqm_spproj_D");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojOp<double, 2>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojOp<double, 3>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojOp<double, 4>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojOp<double, 8>>("DN_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeqm_spproj_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeqm_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeqm_spproj_pD");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpprojOp<double, 2>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpprojOp<double, 3>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpprojOp<double, 4>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpprojOp<double, 8>>("DN_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeqm_spproj_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

}  // extern "C"
