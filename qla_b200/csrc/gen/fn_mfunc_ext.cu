// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA FN mfunc_ext entry points (extern "C"), reference: lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_mfunc_nc2.cuh"

extern "C" {
QLAB_EXPORT void QLA_FN_M_veq_invsqrt_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_invsqrt_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_INVSQRT>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMfuncExtOp<float, 3, 0>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 0>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 0>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_invsqrt_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_log_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_log_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_LOG>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMfuncExtOp<float, 3, 1>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 1>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 1>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_log_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_expA_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_expA_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EXPA>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::ExpAHOp<float, true>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 2>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 2>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_expA_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_expTA_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_expTA_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EXPTA>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::ExpAHOp<float, false>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 2>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 2>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_expTA_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_sqrtPH_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_sqrtPH_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_SQRTPH>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::SqrtPHOp<float, false>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 3>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 3>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_sqrtPH_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_invsqrtPH_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_invsqrtPH_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_INVSQRTPH>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::SqrtPHOp<float, true>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 4>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 4>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_invsqrtPH_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veq_eigenvals_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_V_veq_eigenvals_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EIG>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::EigenvalsOp<float>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenEigenOp<float, 4, false>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenEigenOp<float, 8, false>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_eigenvals_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veq_eigenvalsH_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_V_veq_eigenvalsH_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EIGH>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::EigenvalsHOp<float>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenEigenOp<float, 4, true>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenEigenOp<float, 8, true>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_eigenvalsH_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_invsqrt_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_invsqrt_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_INVSQRT>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMfuncExtOp<float, 3, 0>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 0>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 0>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_invsqrt_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_log_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_log_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_LOG>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMfuncExtOp<float, 3, 1>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 1>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 1>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_log_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_expA_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_expA_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EXPA>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::ExpAHOp<float, true>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 2>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 2>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_expA_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_expTA_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_expTA_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EXPTA>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::ExpAHOp<float, false>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 2>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 2>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_expTA_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_sqrtPH_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_sqrtPH_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_SQRTPH>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::SqrtPHOp<float, false>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 3>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 3>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_sqrtPH_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_invsqrtPH_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_invsqrtPH_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_INVSQRTPH>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::SqrtPHOp<float, true>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 4>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 4>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_invsqrtPH_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veq_eigenvals_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_V_veq_eigenvals_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EIG>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::EigenvalsOp<float>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenEigenOp<float, 4, false>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenEigenOp<float, 8, false>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_eigenvals_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veq_eigenvalsH_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_V_veq_eigenvalsH_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EIGH>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::EigenvalsHOp<float>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenEigenOp<float, 4, true>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenEigenOp<float, 8, true>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_eigenvalsH_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veq_M_inverse_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veq_M_inverse_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MInverseOp<float, 1>>("FN_minv", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMInverseOp<float, 3, 1>>("FN_minv", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMInverseOp<float, 4, 1>>("FN_minv", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMInverseOp<float, 8, 1>>("FN_minv", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_M_inverse_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veq_M_inverse_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veq_M_inverse_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MInverseOp<float, 1>>("FN_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMInverseOp<float, 3, 1>>("FN_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMInverseOp<float, 4, 1>>("FN_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMInverseOp<float, 8, 1>>("FN_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_M_inverse_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veq_pM_inverse_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veq_pM_inverse_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MInverseOp<float, 1>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMInverseOp<float, 3, 1>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMInverseOp<float, 4, 1>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMInverseOp<float, 8, 1>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_pM_inverse_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veq_pM_inverse_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veq_pM_inverse_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MInverseOp<float, 1>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMInverseOp<float, 3, 1>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMInverseOp<float, 4, 1>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMInverseOp<float, 8, 1>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_pM_inverse_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_M_inverse_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_M_inverse_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MInverseOp<float, 2>>("FN_minv", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMInverseOp<float, 3, 3>>("FN_minv", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMInverseOp<float, 4, 4>>("FN_minv", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMInverseOp<float, 8, 8>>("FN_minv", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_M_inverse_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_M_inverse_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_M_inverse_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MInverseOp<float, 2>>("FN_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMInverseOp<float, 3, 3>>("FN_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMInverseOp<float, 4, 4>>("FN_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMInverseOp<float, 8, 8>>("FN_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_M_inverse_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_pM_inverse_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pM_inverse_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MInverseOp<float, 2>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMInverseOp<float, 3, 3>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMInverseOp<float, 4, 4>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMInverseOp<float, 8, 8>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_pM_inverse_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_pM_inverse_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pM_inverse_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MInverseOp<float, 2>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMInverseOp<float, 3, 3>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMInverseOp<float, 4, 4>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMInverseOp<float, 8, 8>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_pM_inverse_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_invsqrt_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_invsqrt_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_INVSQRT>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMfuncExtOp<float, 3, 0>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 0>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 0>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_invsqrt_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_log_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_log_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_LOG>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMfuncExtOp<float, 3, 1>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 1>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 1>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_log_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_expA_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_expA_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EXPA>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::ExpAHOp<float, true>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 2>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 2>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_expA_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_expTA_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_expTA_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EXPTA>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::ExpAHOp<float, false>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 2>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 2>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_expTA_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_sqrtPH_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_sqrtPH_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_SQRTPH>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::SqrtPHOp<float, false>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 3>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 3>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_sqrtPH_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_invsqrtPH_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_invsqrtPH_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_INVSQRTPH>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::SqrtPHOp<float, true>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 4>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 4>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_invsqrtPH_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_eigenvals_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_eigenvals_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EIG>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::EigenvalsOp<float>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenEigenOp<float, 4, false>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenEigenOp<float, 8, false>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_eigenvals_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_eigenvalsH_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_eigenvalsH_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EIGH>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::EigenvalsHOp<float>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenEigenOp<float, 4, true>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenEigenOp<float, 8, true>>("FN_mfunc_ext", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_eigenvalsH_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_invsqrt_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_invsqrt_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_INVSQRT>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMfuncExtOp<float, 3, 0>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 0>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 0>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_invsqrt_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_log_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_log_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_LOG>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMfuncExtOp<float, 3, 1>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 1>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 1>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_log_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_expA_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_expA_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EXPA>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::ExpAHOp<float, true>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 2>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 2>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_expA_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_expTA_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_expTA_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EXPTA>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::ExpAHOp<float, false>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 2>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 2>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_expTA_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_sqrtPH_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_sqrtPH_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_SQRTPH>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::SqrtPHOp<float, false>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 3>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 3>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_sqrtPH_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_invsqrtPH_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_invsqrtPH_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_INVSQRTPH>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::SqrtPHOp<float, true>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMfuncExtOp<float, 4, 4>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMfuncExtOp<float, 8, 4>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_invsqrtPH_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_eigenvals_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_eigenvals_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EIG>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::EigenvalsOp<float>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenEigenOp<float, 4, false>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenEigenOp<float, 8, false>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_eigenvals_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_eigenvalsH_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_eigenvalsH_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EIGH>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::EigenvalsHOp<float>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenEigenOp<float, 4, true>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenEigenOp<float, 8, true>>("FN_mfunc_ext", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_eigenvalsH_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_M_inverse_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_M_inverse_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MInverseOp<float, 1>>("FN_minv", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMInverseOp<float, 3, 1>>("FN_minv", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMInverseOp<float, 4, 1>>("FN_minv", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMInverseOp<float, 8, 1>>("FN_minv", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_M_inverse_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_M_inverse_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_M_inverse_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MInverseOp<float, 1>>("FN_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMInverseOp<float, 3, 1>>("FN_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMInverseOp<float, 4, 1>>("FN_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMInverseOp<float, 8, 1>>("FN_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_M_inverse_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_pM_inverse_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_pM_inverse_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MInverseOp<float, 1>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMInverseOp<float, 3, 1>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMInverseOp<float, 4, 1>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMInverseOp<float, 8, 1>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_pM_inverse_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_pM_inverse_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_pM_inverse_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MInverseOp<float, 1>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMInverseOp<float, 3, 1>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMInverseOp<float, 4, 1>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMInverseOp<float, 8, 1>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_pM_inverse_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_M_inverse_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_M_inverse_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MInverseOp<float, 2>>("FN_minv", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMInverseOp<float, 3, 3>>("FN_minv", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMInverseOp<float, 4, 4>>("FN_minv", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMInverseOp<float, 8, 8>>("FN_minv", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_M_inverse_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_M_inverse_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_M_inverse_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MInverseOp<float, 2>>("FN_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMInverseOp<float, 3, 3>>("FN_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMInverseOp<float, 4, 4>>("FN_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMInverseOp<float, 8, 8>>("FN_minv", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_M_inverse_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_pM_inverse_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pM_inverse_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MInverseOp<float, 2>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMInverseOp<float, 3, 3>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMInverseOp<float, 4, 4>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMInverseOp<float, 8, 8>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_pM_inverse_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_pM_inverse_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pM_inverse_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MInverseOp<float, 2>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenMInverseOp<float, 3, 3>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenMInverseOp<float, 4, 4>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenMInverseOp<float, 8, 8>>("FN_minv", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_pM_inverse_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

}  // extern "C"
