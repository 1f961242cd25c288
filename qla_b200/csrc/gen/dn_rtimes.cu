// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA DN rtimes entry points (extern "C"), reference: lib/perl/build_qla.pl:1256-1292 (real constant times field)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_DN_V_veq_r_times_V(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_V_veq_r_times_V");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 3>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_V_veq_r_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_V_veq_r_times_pV(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_V_veq_r_times_pV");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 3>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_V_veq_r_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_V_vpeq_r_times_V(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_V_vpeq_r_times_V");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 3>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_V_vpeq_r_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_V_vpeq_r_times_pV(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_V_vpeq_r_times_pV");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 3>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_V_vpeq_r_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_V_vmeq_r_times_V(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_V_vmeq_r_times_V");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 3>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_V_vmeq_r_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_V_vmeq_r_times_pV(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_V_vmeq_r_times_pV");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 3>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_V_vmeq_r_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_V_veqm_r_times_V(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_V_veqm_r_times_V");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 3>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_V_veqm_r_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_V_veqm_r_times_pV(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_V_veqm_r_times_pV");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 3>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_V_veqm_r_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_V_xeq_r_times_V(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_V_xeq_r_times_V");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 3>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_V_xeq_r_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_V_xeq_r_times_pV(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_V_xeq_r_times_pV");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 3>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_V_xeq_r_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_V_xpeq_r_times_V(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_V_xpeq_r_times_V");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 3>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_V_xpeq_r_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_V_xpeq_r_times_pV(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_V_xpeq_r_times_pV");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 3>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_V_xpeq_r_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_V_xmeq_r_times_V(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_V_xmeq_r_times_V");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 3>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_V_xmeq_r_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_V_xmeq_r_times_pV(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_V_xmeq_r_times_pV");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 3>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_V_xmeq_r_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_V_xeqm_r_times_V(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_V_xeqm_r_times_V");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 3>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_V_xeqm_r_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_V_xeqm_r_times_pV(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_V_xeqm_r_times_pV");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 3>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_V_xeqm_r_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veq_r_times_H(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_H_veq_r_times_H");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 6>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veq_r_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veq_r_times_pH(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_H_veq_r_times_pH");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 6>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veq_r_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vpeq_r_times_H(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_H_vpeq_r_times_H");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 6>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vpeq_r_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vpeq_r_times_pH(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_H_vpeq_r_times_pH");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 6>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vpeq_r_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vmeq_r_times_H(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_H_vmeq_r_times_H");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 6>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vmeq_r_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_vmeq_r_times_pH(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_H_vmeq_r_times_pH");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 6>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_vmeq_r_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veqm_r_times_H(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_H_veqm_r_times_H");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 6>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veqm_r_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_veqm_r_times_pH(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_H_veqm_r_times_pH");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 6>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_veqm_r_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeq_r_times_H(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeq_r_times_H");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 6>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeq_r_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeq_r_times_pH(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeq_r_times_pH");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 6>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeq_r_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xpeq_r_times_H(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xpeq_r_times_H");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 6>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xpeq_r_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xpeq_r_times_pH(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xpeq_r_times_pH");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 6>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xpeq_r_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xmeq_r_times_H(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xmeq_r_times_H");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 6>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xmeq_r_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xmeq_r_times_pH(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xmeq_r_times_pH");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 6>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xmeq_r_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeqm_r_times_H(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeqm_r_times_H");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 6>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeqm_r_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_H_xeqm_r_times_pH(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_H_xeqm_r_times_pH");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 6>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_H_xeqm_r_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_r_times_D(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_D_veq_r_times_D");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 12>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 32>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_r_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veq_r_times_pD(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_D_veq_r_times_pD");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 12>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 32>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veq_r_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_r_times_D(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_r_times_D");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 12>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 32>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_r_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vpeq_r_times_pD(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_D_vpeq_r_times_pD");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 12>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 32>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vpeq_r_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_r_times_D(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_r_times_D");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 12>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 32>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_r_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_vmeq_r_times_pD(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_D_vmeq_r_times_pD");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 12>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 32>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_vmeq_r_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_r_times_D(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_r_times_D");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 12>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 32>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_r_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_veqm_r_times_pD(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_D_veqm_r_times_pD");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 12>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 32>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_veqm_r_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_r_times_D(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_r_times_D");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 12>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 32>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_r_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeq_r_times_pD(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeq_r_times_pD");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 12>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 32>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeq_r_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_r_times_D(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_r_times_D");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 12>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 32>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_r_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xpeq_r_times_pD(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xpeq_r_times_pD");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 12>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 32>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xpeq_r_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_r_times_D(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_r_times_D");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 12>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 32>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_r_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xmeq_r_times_pD(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xmeq_r_times_pD");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 12>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 32>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xmeq_r_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_r_times_D(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_r_times_D");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 12>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 32>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_r_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_D_xeqm_r_times_pD(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_D_xeqm_r_times_pD");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 12>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 32>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_D_xeqm_r_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_veq_r_times_M(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_M_veq_r_times_M");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 9>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 64>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_veq_r_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_veq_r_times_pM(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_M_veq_r_times_pM");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 9>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 64>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_veq_r_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_vpeq_r_times_M(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_M_vpeq_r_times_M");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 9>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 64>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_vpeq_r_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_vpeq_r_times_pM(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_M_vpeq_r_times_pM");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 9>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 64>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_vpeq_r_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_vmeq_r_times_M(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_M_vmeq_r_times_M");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 9>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 64>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_vmeq_r_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_vmeq_r_times_pM(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_M_vmeq_r_times_pM");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 9>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 64>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_vmeq_r_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_veqm_r_times_M(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_M_veqm_r_times_M");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 9>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 64>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_veqm_r_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_veqm_r_times_pM(int nc, void * r, QLA_D_Real * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_M_veqm_r_times_pM");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 9>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 64>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_veqm_r_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_xeq_r_times_M(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeq_r_times_M");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 9>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 64>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_xeq_r_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_xeq_r_times_pM(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeq_r_times_pM");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 9>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 64>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_xeq_r_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_xpeq_r_times_M(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xpeq_r_times_M");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 9>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 64>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_xpeq_r_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_xpeq_r_times_pM(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xpeq_r_times_pM");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 9>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 64>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_xpeq_r_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_xmeq_r_times_M(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xmeq_r_times_M");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 9>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 64>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_xmeq_r_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_xmeq_r_times_pM(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xmeq_r_times_pM");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 9>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 64>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_xmeq_r_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_xeqm_r_times_M(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeqm_r_times_M");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 9>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 64>, double>("DN_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_xeqm_r_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_xeqm_r_times_pM(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeqm_r_times_pM");
  switch (nc) {
    case 2: qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_scalar_map<qlab::RTimesOp<double, 9>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_scalar_map<qlab::RTimesOp<double, 16>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_scalar_map<qlab::RTimesOp<double, 64>, double>("DN_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_xeqm_r_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

}  // extern "C"
