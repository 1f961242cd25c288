// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA DN dot entry points (extern "C"), reference: lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_DN_c_veq_V_dot_V(int nc, QLA_D_Complex * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_V_dot_V");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 2, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 3, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_veq_V_dot_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_veq_V_dot_pV(int nc, QLA_D_Complex * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_V_dot_pV");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 2, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 3, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_veq_V_dot_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_veq_pV_dot_V(int nc, QLA_D_Complex * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_pV_dot_V");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 2, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 3, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_veq_pV_dot_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_veq_pV_dot_pV(int nc, QLA_D_Complex * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_pV_dot_pV");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 2, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 3, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_veq_pV_dot_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_xeq_V_dot_V(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_V_dot_V");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 2, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 3, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_xeq_V_dot_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_xeq_V_dot_pV(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_V_dot_pV");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 2, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 3, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_xeq_V_dot_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_xeq_pV_dot_V(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_pV_dot_V");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 2, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 3, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_xeq_pV_dot_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_xeq_pV_dot_pV(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_pV_dot_pV");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 2, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 3, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_xeq_pV_dot_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_veq_H_dot_H(int nc, QLA_D_Complex * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_H_dot_H");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 6, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_veq_H_dot_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_veq_H_dot_pH(int nc, QLA_D_Complex * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_H_dot_pH");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 6, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_veq_H_dot_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_veq_pH_dot_H(int nc, QLA_D_Complex * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_pH_dot_H");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 6, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_veq_pH_dot_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_veq_pH_dot_pH(int nc, QLA_D_Complex * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_pH_dot_pH");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 6, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_veq_pH_dot_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_xeq_H_dot_H(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_H_dot_H");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 6, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_xeq_H_dot_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_xeq_H_dot_pH(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_H_dot_pH");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 6, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_xeq_H_dot_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_xeq_pH_dot_H(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_pH_dot_H");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 6, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_xeq_pH_dot_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_xeq_pH_dot_pH(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_pH_dot_pH");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 6, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_xeq_pH_dot_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_veq_D_dot_D(int nc, QLA_D_Complex * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_D_dot_D");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 12, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 32, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_veq_D_dot_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_veq_D_dot_pD(int nc, QLA_D_Complex * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_D_dot_pD");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 12, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 32, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_veq_D_dot_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_veq_pD_dot_D(int nc, QLA_D_Complex * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_pD_dot_D");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 12, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 32, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_veq_pD_dot_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_veq_pD_dot_pD(int nc, QLA_D_Complex * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_pD_dot_pD");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 12, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 32, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_veq_pD_dot_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_xeq_D_dot_D(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_D_dot_D");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 12, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 32, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_xeq_D_dot_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_xeq_D_dot_pD(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_D_dot_pD");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 12, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 32, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_xeq_D_dot_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_xeq_pD_dot_D(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_pD_dot_D");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 12, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 32, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_xeq_pD_dot_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_xeq_pD_dot_pD(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_pD_dot_pD");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 8, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 12, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 32, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_xeq_pD_dot_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_veq_M_dot_M(int nc, QLA_D_Complex * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_M_dot_M");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 9, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 64, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_veq_M_dot_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_veq_M_dot_pM(int nc, QLA_D_Complex * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_M_dot_pM");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 9, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 64, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_veq_M_dot_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_veq_pM_dot_M(int nc, QLA_D_Complex * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_pM_dot_M");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 9, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 64, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_veq_pM_dot_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_veq_pM_dot_pM(int nc, QLA_D_Complex * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_DN_c_veq_pM_dot_pM");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 9, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 64, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_veq_pM_dot_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_xeq_M_dot_M(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_M_dot_M");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 9, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 64, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_xeq_M_dot_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_xeq_M_dot_pM(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_M_dot_pM");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 9, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 64, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_xeq_M_dot_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_xeq_pM_dot_M(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_pM_dot_M");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 9, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 64, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_xeq_pM_dot_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_c_xeq_pM_dot_pM(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_DN_c_xeq_pM_dot_pM");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::DotOp<double, 4, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 3: qlab::api_reduce<qlab::DotOp<double, 9, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 4: qlab::api_reduce<qlab::DotOp<double, 16, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n); break;
    case 8: qlab::api_reduce<qlab::DotOp<double, 64, double>>("DN_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_c_xeq_pM_dot_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

}  // extern "C"
