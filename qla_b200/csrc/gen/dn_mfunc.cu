// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA DN mfunc entry points (extern "C"), reference: lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_mfunc_nc2.cuh"

extern "C" {
QLAB_EXPORT void QLA_DN_M_veq_exp_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_M_veq_exp_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EXP>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenExpOp<double, 3>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenExpOp<double, 4>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenExpOp<double, 8>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_veq_exp_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_veq_sqrt_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_M_veq_sqrt_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_SQRT>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenSqrtOp<double, 3>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenSqrtOp<double, 4>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenSqrtOp<double, 8>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_veq_sqrt_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_veq_inverse_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_M_veq_inverse_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_INVERSE>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenInverseOp<double, 3>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenInverseOp<double, 4>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenInverseOp<double, 8>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_veq_inverse_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_C_veq_det_M(int nc, QLA_D_Complex * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_C_veq_det_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_DET>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenDetOp<double, 3>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenDetOp<double, 4>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenDetOp<double, 8>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_C_veq_det_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_veq_exp_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_M_veq_exp_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EXP>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenExpOp<double, 3>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenExpOp<double, 4>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenExpOp<double, 8>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_veq_exp_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_veq_sqrt_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_M_veq_sqrt_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_SQRT>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenSqrtOp<double, 3>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenSqrtOp<double, 4>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenSqrtOp<double, 8>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_veq_sqrt_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_veq_inverse_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_M_veq_inverse_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_INVERSE>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenInverseOp<double, 3>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenInverseOp<double, 4>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenInverseOp<double, 8>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_veq_inverse_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_C_veq_det_pM(int nc, QLA_D_Complex * r, void * a, int n) {
  QLAB_TRACE("QLA_DN_C_veq_det_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_DET>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenDetOp<double, 3>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenDetOp<double, 4>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenDetOp<double, 8>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_C_veq_det_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_xeq_exp_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeq_exp_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EXP>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenExpOp<double, 3>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenExpOp<double, 4>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenExpOp<double, 8>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_xeq_exp_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_xeq_sqrt_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeq_sqrt_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_SQRT>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenSqrtOp<double, 3>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenSqrtOp<double, 4>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenSqrtOp<double, 8>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_xeq_sqrt_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_xeq_inverse_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeq_inverse_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_INVERSE>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenInverseOp<double, 3>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenInverseOp<double, 4>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenInverseOp<double, 8>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_xeq_inverse_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_C_xeq_det_M(int nc, QLA_D_Complex * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_C_xeq_det_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_DET>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenDetOp<double, 3>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenDetOp<double, 4>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenDetOp<double, 8>>("DN_mfunc", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_C_xeq_det_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_xeq_exp_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeq_exp_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_EXP>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenExpOp<double, 3>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenExpOp<double, 4>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenExpOp<double, 8>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_xeq_exp_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_xeq_sqrt_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeq_sqrt_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_SQRT>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenSqrtOp<double, 3>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenSqrtOp<double, 4>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenSqrtOp<double, 8>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_xeq_sqrt_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_M_xeq_inverse_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_M_xeq_inverse_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_INVERSE>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenInverseOp<double, 3>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenInverseOp<double, 4>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenInverseOp<double, 8>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_M_xeq_inverse_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_DN_C_xeq_det_pM(int nc, QLA_D_Complex * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_DN_C_xeq_det_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::Nc2MfuncOp<double, qlab::N2_DET>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::GenDetOp<double, 3>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::GenDetOp<double, 4>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::GenDetOp<double, 8>>("DN_mfunc", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_DN_C_xeq_det_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

}  // extern "C"
