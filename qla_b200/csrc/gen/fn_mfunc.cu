// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA FN mfunc entry points (extern "C"), reference: lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_mfunc_nc2.cuh"

extern "C" {
QLAB_EXPORT void QLA_FN_M_veq_exp_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_exp_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EXP>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenExpOp<float, 3>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenExpOp<float, 4>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenExpOp<float, 8>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_exp_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_sqrt_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_sqrt_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_SQRT>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenSqrtOp<float, 3>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenSqrtOp<float, 4>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenSqrtOp<float, 8>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_sqrt_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_inverse_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_inverse_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_INVERSE>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenInverseOp<float, 3>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenInverseOp<float, 4>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenInverseOp<float, 8>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_inverse_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_C_veq_det_M(int nc, QLA_F_Complex * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_C_veq_det_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_DET>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenDetOp<float, 3>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenDetOp<float, 4>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenDetOp<float, 8>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_C_veq_det_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_exp_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_exp_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EXP>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenExpOp<float, 3>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenExpOp<float, 4>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenExpOp<float, 8>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_exp_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_sqrt_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_sqrt_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_SQRT>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenSqrtOp<float, 3>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenSqrtOp<float, 4>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenSqrtOp<float, 8>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_sqrt_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_inverse_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_inverse_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_INVERSE>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenInverseOp<float, 3>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenInverseOp<float, 4>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenInverseOp<float, 8>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_inverse_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_C_veq_det_pM(int nc, QLA_F_Complex * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_C_veq_det_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_DET>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenDetOp<float, 3>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenDetOp<float, 4>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenDetOp<float, 8>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_C_veq_det_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_exp_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_exp_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EXP>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenExpOp<float, 3>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenExpOp<float, 4>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenExpOp<float, 8>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_exp_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_sqrt_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_sqrt_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_SQRT>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenSqrtOp<float, 3>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenSqrtOp<float, 4>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenSqrtOp<float, 8>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_sqrt_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_inverse_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_inverse_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_INVERSE>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenInverseOp<float, 3>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenInverseOp<float, 4>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenInverseOp<float, 8>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_inverse_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_C_xeq_det_M(int nc, QLA_F_Complex * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_C_xeq_det_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_DET>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenDetOp<float, 3>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenDetOp<float, 4>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenDetOp<float, 8>>("FN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_C_xeq_det_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_exp_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_exp_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_EXP>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenExpOp<float, 3>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenExpOp<float, 4>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenExpOp<float, 8>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_exp_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_sqrt_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_sqrt_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_SQRT>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenSqrtOp<float, 3>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenSqrtOp<float, 4>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenSqrtOp<float, 8>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_sqrt_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_inverse_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_inverse_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_INVERSE>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenInverseOp<float, 3>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenInverseOp<float, 4>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenInverseOp<float, 8>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_inverse_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_C_xeq_det_pM(int nc, QLA_F_Complex * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_C_xeq_det_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<float, qlab::N2_DET>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenDetOp<float, 3>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenDetOp<float, 4>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenDetOp<float, 8>>("FN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_C_xeq_det_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

}  // extern "C"
