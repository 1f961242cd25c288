// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA FN norm2 entry points (extern "C"), reference: lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_FN_r_veq_norm2_V(int nc, QLA_F_Real * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_r_veq_norm2_V");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 2, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 3, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 4, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 8, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_r_veq_norm2_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_r_veq_norm2_pV(int nc, QLA_F_Real * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_r_veq_norm2_pV");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 2, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 3, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 4, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 8, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_r_veq_norm2_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_r_xeq_norm2_V(int nc, QLA_F_Real * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_r_xeq_norm2_V");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 2, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 3, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 4, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 8, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_r_xeq_norm2_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_r_xeq_norm2_pV(int nc, QLA_F_Real * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_r_xeq_norm2_pV");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 2, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 3, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 4, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 8, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_r_xeq_norm2_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DFN_r_veq_norm2_V(int nc, QLA_D_Real * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_r_veq_norm2_V");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 2, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 3, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 4, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 8, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DFN_r_veq_norm2_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DFN_r_veq_norm2_pV(int nc, QLA_D_Real * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_r_veq_norm2_pV");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 2, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 3, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 4, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 8, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DFN_r_veq_norm2_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DFN_r_xeq_norm2_V(int nc, QLA_D_Real * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_r_xeq_norm2_V");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 2, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 3, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 4, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 8, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DFN_r_xeq_norm2_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DFN_r_xeq_norm2_pV(int nc, QLA_D_Real * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_r_xeq_norm2_pV");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 2, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 3, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 4, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 8, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DFN_r_xeq_norm2_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_r_veq_norm2_H(int nc, QLA_F_Real * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_r_veq_norm2_H");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 4, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 6, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 8, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 16, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_r_veq_norm2_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_r_veq_norm2_pH(int nc, QLA_F_Real * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_r_veq_norm2_pH");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 4, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 6, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 8, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 16, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_r_veq_norm2_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_r_xeq_norm2_H(int nc, QLA_F_Real * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_r_xeq_norm2_H");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 4, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 6, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 8, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 16, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_r_xeq_norm2_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_r_xeq_norm2_pH(int nc, QLA_F_Real * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_r_xeq_norm2_pH");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 4, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 6, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 8, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 16, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_r_xeq_norm2_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DFN_r_veq_norm2_H(int nc, QLA_D_Real * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_r_veq_norm2_H");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 4, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 6, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 8, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 16, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DFN_r_veq_norm2_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DFN_r_veq_norm2_pH(int nc, QLA_D_Real * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_r_veq_norm2_pH");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 4, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 6, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 8, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 16, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DFN_r_veq_norm2_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DFN_r_xeq_norm2_H(int nc, QLA_D_Real * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_r_xeq_norm2_H");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 4, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 6, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 8, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 16, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DFN_r_xeq_norm2_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DFN_r_xeq_norm2_pH(int nc, QLA_D_Real * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_r_xeq_norm2_pH");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 4, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 6, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 8, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 16, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DFN_r_xeq_norm2_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_r_veq_norm2_D(int nc, QLA_F_Real * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_r_veq_norm2_D");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 8, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 12, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 16, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 32, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_r_veq_norm2_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_r_veq_norm2_pD(int nc, QLA_F_Real * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_r_veq_norm2_pD");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 8, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 12, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 16, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 32, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_r_veq_norm2_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_r_xeq_norm2_D(int nc, QLA_F_Real * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_r_xeq_norm2_D");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 8, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 12, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 16, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 32, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_r_xeq_norm2_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_r_xeq_norm2_pD(int nc, QLA_F_Real * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_r_xeq_norm2_pD");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 8, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 12, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 16, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 32, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_r_xeq_norm2_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DFN_r_veq_norm2_D(int nc, QLA_D_Real * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_r_veq_norm2_D");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 8, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 12, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 16, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 32, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DFN_r_veq_norm2_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DFN_r_veq_norm2_pD(int nc, QLA_D_Real * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_r_veq_norm2_pD");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 8, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 12, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 16, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 32, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DFN_r_veq_norm2_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DFN_r_xeq_norm2_D(int nc, QLA_D_Real * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_r_xeq_norm2_D");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 8, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 12, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 16, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 32, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DFN_r_xeq_norm2_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DFN_r_xeq_norm2_pD(int nc, QLA_D_Real * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_r_xeq_norm2_pD");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 8, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 12, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 16, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 32, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DFN_r_xeq_norm2_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_r_veq_norm2_M(int nc, QLA_F_Real * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_r_veq_norm2_M");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 4, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 9, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 16, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 64, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_r_veq_norm2_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_r_veq_norm2_pM(int nc, QLA_F_Real * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_r_veq_norm2_pM");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 4, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 9, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 16, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 64, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_r_veq_norm2_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_r_xeq_norm2_M(int nc, QLA_F_Real * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_r_xeq_norm2_M");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 4, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 9, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 16, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 64, float>>("FN_norm2", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_r_xeq_norm2_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_r_xeq_norm2_pM(int nc, QLA_F_Real * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_r_xeq_norm2_pM");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 4, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 9, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 16, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 64, float>>("FN_norm2", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_r_xeq_norm2_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DFN_r_veq_norm2_M(int nc, QLA_D_Real * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_r_veq_norm2_M");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 4, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 9, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 16, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 64, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DFN_r_veq_norm2_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DFN_r_veq_norm2_pM(int nc, QLA_D_Real * r, void * a, int n) {
  QLAB_TRACE("QLA_DFN_r_veq_norm2_pM");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 4, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 9, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 16, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 64, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DFN_r_veq_norm2_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DFN_r_xeq_norm2_M(int nc, QLA_D_Real * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_r_xeq_norm2_M");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 4, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 9, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 16, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 64, double>>("FN_norm2", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DFN_r_xeq_norm2_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DFN_r_xeq_norm2_pM(int nc, QLA_D_Real * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DFN_r_xeq_norm2_pM");
  switch (nc) {
    case 2: qlab::api_reduce<qlab::Norm2Op<float, 4, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 3: qlab::api_reduce<qlab::Norm2Op<float, 9, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 4: qlab::api_reduce<qlab::Norm2Op<float, 16, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    case 8: qlab::api_reduce<qlab::Norm2Op<float, 64, double>>("FN_norm2", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DFN_r_xeq_norm2_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

}  // extern "C"
