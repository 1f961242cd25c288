// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA DN sprecon entry points (extern "C"), reference: lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_DN_D_veq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_sprecon_H");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconOp<double, 2>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconOp<double, 3>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconOp<double, 4>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconOp<double, 8>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_sprecon_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veq_sprecon_pH");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconOp<double, 2>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconOp<double, 3>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconOp<double, 4>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconOp<double, 8>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_sprecon_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_sprecon_H");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconOp<double, 2>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconOp<double, 3>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconOp<double, 4>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconOp<double, 8>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_sprecon_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_sprecon_pH");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconOp<double, 2>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconOp<double, 3>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconOp<double, 4>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconOp<double, 8>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_sprecon_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_sprecon_H");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconOp<double, 2>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconOp<double, 3>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconOp<double, 4>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconOp<double, 8>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_sprecon_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_sprecon_pH");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconOp<double, 2>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconOp<double, 3>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconOp<double, 4>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconOp<double, 8>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_sprecon_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_sprecon_H(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_sprecon_H");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconOp<double, 2>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconOp<double, 3>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconOp<double, 4>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconOp<double, 8>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_sprecon_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_sprecon_pH");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconOp<double, 2>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconOp<double, 3>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconOp<double, 4>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconOp<double, 8>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_sprecon_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_sprecon_H");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconOp<double, 2>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconOp<double, 3>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconOp<double, 4>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconOp<double, 8>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_sprecon_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_sprecon_pH");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconOp<double, 2>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconOp<double, 3>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconOp<double, 4>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconOp<double, 8>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_sprecon_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_sprecon_H");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconOp<double, 2>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconOp<double, 3>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconOp<double, 4>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconOp<double, 8>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_sprecon_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_sprecon_pH");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconOp<double, 2>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconOp<double, 3>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconOp<double, 4>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconOp<double, 8>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_sprecon_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_sprecon_H");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconOp<double, 2>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconOp<double, 3>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconOp<double, 4>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconOp<double, 8>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_sprecon_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_sprecon_pH");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconOp<double, 2>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconOp<double, 3>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconOp<double, 4>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconOp<double, 8>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_sprecon_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_sprecon_H(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_sprecon_H");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconOp<double, 2>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconOp<double, 3>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconOp<double, 4>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconOp<double, 8>>("DN_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_sprecon_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_sprecon_pH");
  if (mu < 0 || mu > 4) return;
  switch (nc) {
    case 2: qlab::api_map<qlab::SpreconOp<double, 2>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 3: qlab::api_map<qlab::SpreconOp<double, 3>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 4: qlab::api_map<qlab::SpreconOp<double, 4>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    case 8: qlab::api_map<qlab::SpreconOp<double, 8>>("DN_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_sprecon_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

}  // extern "C"
