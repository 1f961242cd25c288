// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA FN lmult entry points (extern "C"), reference: lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_FN_V_veq_M_times_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veq_M_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_M_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veq_M_times_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veq_M_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_M_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veq_Ma_times_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veq_Ma_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_Ma_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veq_Ma_times_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veq_Ma_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_Ma_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veq_pM_times_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veq_pM_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_pM_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veq_pM_times_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veq_pM_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_pM_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veq_pMa_times_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veq_pMa_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_pMa_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veq_pMa_times_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veq_pMa_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_pMa_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vpeq_M_times_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_vpeq_M_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vpeq_M_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vpeq_M_times_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_vpeq_M_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vpeq_M_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vpeq_Ma_times_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_vpeq_Ma_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vpeq_Ma_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vpeq_Ma_times_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_vpeq_Ma_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vpeq_Ma_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vpeq_pM_times_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_vpeq_pM_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vpeq_pM_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vpeq_pM_times_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_vpeq_pM_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vpeq_pM_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vpeq_pMa_times_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_vpeq_pMa_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vpeq_pMa_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vpeq_pMa_times_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_vpeq_pMa_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vpeq_pMa_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vmeq_M_times_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_vmeq_M_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vmeq_M_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vmeq_M_times_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_vmeq_M_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vmeq_M_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vmeq_Ma_times_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_vmeq_Ma_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vmeq_Ma_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vmeq_Ma_times_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_vmeq_Ma_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vmeq_Ma_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vmeq_pM_times_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_vmeq_pM_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vmeq_pM_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vmeq_pM_times_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_vmeq_pM_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vmeq_pM_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vmeq_pMa_times_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_vmeq_pMa_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vmeq_pMa_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vmeq_pMa_times_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_vmeq_pMa_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vmeq_pMa_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veqm_M_times_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veqm_M_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veqm_M_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veqm_M_times_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veqm_M_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veqm_M_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veqm_Ma_times_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veqm_Ma_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veqm_Ma_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veqm_Ma_times_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veqm_Ma_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veqm_Ma_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veqm_pM_times_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veqm_pM_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veqm_pM_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veqm_pM_times_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veqm_pM_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veqm_pM_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veqm_pMa_times_V(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veqm_pMa_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veqm_pMa_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veqm_pMa_times_pV(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_V_veqm_pMa_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veqm_pMa_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_M_times_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_M_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_M_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_M_times_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_M_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_M_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_Ma_times_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_Ma_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_Ma_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_Ma_times_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_Ma_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_Ma_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_pM_times_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_pM_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_pM_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_pM_times_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_pM_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_pM_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_pMa_times_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_pMa_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_pMa_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_pMa_times_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_pMa_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_pMa_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xpeq_M_times_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xpeq_M_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xpeq_M_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xpeq_M_times_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xpeq_M_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xpeq_M_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xpeq_Ma_times_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xpeq_Ma_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xpeq_Ma_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xpeq_Ma_times_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xpeq_Ma_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xpeq_Ma_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xpeq_pM_times_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xpeq_pM_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xpeq_pM_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xpeq_pM_times_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xpeq_pM_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xpeq_pM_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xpeq_pMa_times_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xpeq_pMa_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xpeq_pMa_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xpeq_pMa_times_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xpeq_pMa_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xpeq_pMa_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xmeq_M_times_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xmeq_M_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xmeq_M_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xmeq_M_times_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xmeq_M_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xmeq_M_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xmeq_Ma_times_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xmeq_Ma_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xmeq_Ma_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xmeq_Ma_times_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xmeq_Ma_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xmeq_Ma_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xmeq_pM_times_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xmeq_pM_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xmeq_pM_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xmeq_pM_times_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xmeq_pM_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xmeq_pM_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xmeq_pMa_times_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xmeq_pMa_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xmeq_pMa_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xmeq_pMa_times_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xmeq_pMa_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xmeq_pMa_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeqm_M_times_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeqm_M_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeqm_M_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeqm_M_times_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeqm_M_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeqm_M_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeqm_Ma_times_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeqm_Ma_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeqm_Ma_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeqm_Ma_times_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeqm_Ma_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeqm_Ma_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeqm_pM_times_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeqm_pM_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeqm_pM_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeqm_pM_times_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeqm_pM_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeqm_pM_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeqm_pMa_times_V(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeqm_pMa_times_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeqm_pMa_times_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeqm_pMa_times_pV(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeqm_pMa_times_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeqm_pMa_times_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_eq_M_times_xV(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_V_eq_M_times_xV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_eq_M_times_xV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_eq_Ma_times_xV(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_V_eq_Ma_times_xV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_eq_Ma_times_xV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_peq_M_times_xV(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_V_peq_M_times_xV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_peq_M_times_xV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_peq_Ma_times_xV(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_V_peq_Ma_times_xV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_peq_Ma_times_xV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_meq_M_times_xV(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_V_meq_M_times_xV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_meq_M_times_xV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_meq_Ma_times_xV(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_V_meq_Ma_times_xV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_meq_Ma_times_xV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_eqm_M_times_xV(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_V_eqm_M_times_xV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_eqm_M_times_xV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_eqm_Ma_times_xV(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_V_eqm_Ma_times_xV");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 1, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_eqm_Ma_times_xV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veq_M_times_H(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_veq_M_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veq_M_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veq_M_times_pH(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_veq_M_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veq_M_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veq_Ma_times_H(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_veq_Ma_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veq_Ma_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veq_Ma_times_pH(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_veq_Ma_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veq_Ma_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veq_pM_times_H(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_veq_pM_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veq_pM_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veq_pM_times_pH(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_veq_pM_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veq_pM_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veq_pMa_times_H(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_veq_pMa_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veq_pMa_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veq_pMa_times_pH(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_veq_pMa_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veq_pMa_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vpeq_M_times_H(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_vpeq_M_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vpeq_M_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vpeq_M_times_pH(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_vpeq_M_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vpeq_M_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vpeq_Ma_times_H(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_vpeq_Ma_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vpeq_Ma_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vpeq_Ma_times_pH(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_vpeq_Ma_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vpeq_Ma_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vpeq_pM_times_H(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_vpeq_pM_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vpeq_pM_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vpeq_pM_times_pH(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_vpeq_pM_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vpeq_pM_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vpeq_pMa_times_H(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_vpeq_pMa_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vpeq_pMa_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vpeq_pMa_times_pH(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_vpeq_pMa_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vpeq_pMa_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vmeq_M_times_H(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_vmeq_M_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vmeq_M_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vmeq_M_times_pH(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_vmeq_M_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vmeq_M_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vmeq_Ma_times_H(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_vmeq_Ma_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vmeq_Ma_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vmeq_Ma_times_pH(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_vmeq_Ma_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vmeq_Ma_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vmeq_pM_times_H(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_vmeq_pM_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vmeq_pM_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vmeq_pM_times_pH(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_vmeq_pM_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vmeq_pM_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vmeq_pMa_times_H(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_vmeq_pMa_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vmeq_pMa_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vmeq_pMa_times_pH(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_vmeq_pMa_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vmeq_pMa_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veqm_M_times_H(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_veqm_M_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veqm_M_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veqm_M_times_pH(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_veqm_M_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veqm_M_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veqm_Ma_times_H(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_veqm_Ma_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veqm_Ma_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veqm_Ma_times_pH(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_veqm_Ma_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veqm_Ma_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veqm_pM_times_H(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_veqm_pM_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veqm_pM_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veqm_pM_times_pH(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_veqm_pM_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veqm_pM_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veqm_pMa_times_H(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_veqm_pMa_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veqm_pMa_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veqm_pMa_times_pH(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_H_veqm_pMa_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veqm_pMa_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeq_M_times_H(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeq_M_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeq_M_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeq_M_times_pH(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeq_M_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeq_M_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeq_Ma_times_H(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeq_Ma_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeq_Ma_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeq_Ma_times_pH(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeq_Ma_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeq_Ma_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeq_pM_times_H(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeq_pM_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeq_pM_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeq_pM_times_pH(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeq_pM_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeq_pM_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeq_pMa_times_H(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeq_pMa_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeq_pMa_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeq_pMa_times_pH(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeq_pMa_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeq_pMa_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xpeq_M_times_H(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xpeq_M_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xpeq_M_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xpeq_M_times_pH(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xpeq_M_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xpeq_M_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xpeq_Ma_times_H(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xpeq_Ma_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xpeq_Ma_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xpeq_Ma_times_pH(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xpeq_Ma_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xpeq_Ma_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xpeq_pM_times_H(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xpeq_pM_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xpeq_pM_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xpeq_pM_times_pH(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xpeq_pM_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xpeq_pM_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xpeq_pMa_times_H(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xpeq_pMa_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xpeq_pMa_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xpeq_pMa_times_pH(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xpeq_pMa_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xpeq_pMa_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xmeq_M_times_H(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xmeq_M_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xmeq_M_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xmeq_M_times_pH(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xmeq_M_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xmeq_M_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xmeq_Ma_times_H(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xmeq_Ma_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xmeq_Ma_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xmeq_Ma_times_pH(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xmeq_Ma_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xmeq_Ma_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xmeq_pM_times_H(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xmeq_pM_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xmeq_pM_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xmeq_pM_times_pH(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xmeq_pM_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xmeq_pM_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xmeq_pMa_times_H(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xmeq_pMa_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xmeq_pMa_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xmeq_pMa_times_pH(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xmeq_pMa_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xmeq_pMa_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeqm_M_times_H(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeqm_M_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeqm_M_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeqm_M_times_pH(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeqm_M_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeqm_M_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeqm_Ma_times_H(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeqm_Ma_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeqm_Ma_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeqm_Ma_times_pH(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeqm_Ma_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeqm_Ma_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeqm_pM_times_H(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeqm_pM_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeqm_pM_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeqm_pM_times_pH(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeqm_pM_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeqm_pM_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeqm_pMa_times_H(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeqm_pMa_times_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeqm_pMa_times_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeqm_pMa_times_pH(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeqm_pMa_times_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeqm_pMa_times_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_eq_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_H_eq_M_times_xH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_eq_M_times_xH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_eq_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_H_eq_Ma_times_xH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_eq_Ma_times_xH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_peq_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_H_peq_M_times_xH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_peq_M_times_xH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_peq_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_H_peq_Ma_times_xH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_peq_Ma_times_xH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_meq_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_H_meq_M_times_xH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_meq_M_times_xH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_meq_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_H_meq_Ma_times_xH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_meq_Ma_times_xH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_eqm_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_H_eqm_M_times_xH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_eqm_M_times_xH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_eqm_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_H_eqm_Ma_times_xH");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_eqm_Ma_times_xH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veq_M_times_D(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_veq_M_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veq_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veq_M_times_pD(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_veq_M_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veq_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veq_Ma_times_D(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_veq_Ma_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veq_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veq_Ma_times_pD(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_veq_Ma_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veq_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veq_pM_times_D(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_veq_pM_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veq_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veq_pM_times_pD(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_veq_pM_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veq_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veq_pMa_times_D(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_veq_pMa_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veq_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veq_pMa_times_pD(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_veq_pMa_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veq_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vpeq_M_times_D(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_vpeq_M_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vpeq_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vpeq_M_times_pD(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_vpeq_M_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vpeq_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vpeq_Ma_times_D(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_vpeq_Ma_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vpeq_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vpeq_Ma_times_pD(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_vpeq_Ma_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vpeq_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vpeq_pM_times_D(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_vpeq_pM_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vpeq_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vpeq_pM_times_pD(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_vpeq_pM_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vpeq_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vpeq_pMa_times_D(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_vpeq_pMa_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vpeq_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vpeq_pMa_times_pD(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_vpeq_pMa_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vpeq_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vmeq_M_times_D(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_vmeq_M_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vmeq_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vmeq_M_times_pD(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_vmeq_M_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vmeq_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vmeq_Ma_times_D(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_vmeq_Ma_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vmeq_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vmeq_Ma_times_pD(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_vmeq_Ma_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vmeq_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vmeq_pM_times_D(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_vmeq_pM_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vmeq_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vmeq_pM_times_pD(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_vmeq_pM_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vmeq_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vmeq_pMa_times_D(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_vmeq_pMa_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vmeq_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vmeq_pMa_times_pD(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_vmeq_pMa_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vmeq_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veqm_M_times_D(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_veqm_M_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veqm_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veqm_M_times_pD(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_veqm_M_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veqm_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veqm_Ma_times_D(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_veqm_Ma_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veqm_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veqm_Ma_times_pD(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_veqm_Ma_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veqm_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veqm_pM_times_D(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_veqm_pM_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veqm_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veqm_pM_times_pD(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_veqm_pM_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veqm_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veqm_pMa_times_D(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_veqm_pMa_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veqm_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veqm_pMa_times_pD(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_D_veqm_pMa_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veqm_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeq_M_times_D(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeq_M_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeq_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeq_M_times_pD(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeq_M_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeq_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeq_Ma_times_D(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeq_Ma_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeq_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeq_Ma_times_pD(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeq_Ma_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeq_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeq_pM_times_D(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeq_pM_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeq_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeq_pM_times_pD(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeq_pM_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeq_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeq_pMa_times_D(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeq_pMa_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeq_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeq_pMa_times_pD(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeq_pMa_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeq_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xpeq_M_times_D(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xpeq_M_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xpeq_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xpeq_M_times_pD(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xpeq_M_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xpeq_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xpeq_Ma_times_D(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xpeq_Ma_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xpeq_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xpeq_Ma_times_pD(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xpeq_Ma_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xpeq_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xpeq_pM_times_D(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xpeq_pM_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xpeq_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xpeq_pM_times_pD(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xpeq_pM_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xpeq_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xpeq_pMa_times_D(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xpeq_pMa_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xpeq_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xpeq_pMa_times_pD(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xpeq_pMa_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xpeq_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xmeq_M_times_D(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xmeq_M_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xmeq_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xmeq_M_times_pD(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xmeq_M_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xmeq_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xmeq_Ma_times_D(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xmeq_Ma_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xmeq_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xmeq_Ma_times_pD(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xmeq_Ma_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xmeq_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xmeq_pM_times_D(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xmeq_pM_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xmeq_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xmeq_pM_times_pD(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xmeq_pM_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xmeq_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xmeq_pMa_times_D(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xmeq_pMa_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xmeq_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xmeq_pMa_times_pD(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xmeq_pMa_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xmeq_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeqm_M_times_D(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeqm_M_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeqm_M_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeqm_M_times_pD(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeqm_M_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeqm_M_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeqm_Ma_times_D(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeqm_Ma_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeqm_Ma_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeqm_Ma_times_pD(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeqm_Ma_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeqm_Ma_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeqm_pM_times_D(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeqm_pM_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeqm_pM_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeqm_pM_times_pD(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeqm_pM_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeqm_pM_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeqm_pMa_times_D(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeqm_pMa_times_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeqm_pMa_times_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeqm_pMa_times_pD(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeqm_pMa_times_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeqm_pMa_times_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_eq_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_D_eq_M_times_xD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_eq_M_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_eq_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_D_eq_Ma_times_xD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_eq_Ma_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_peq_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_D_peq_M_times_xD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_peq_M_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_peq_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_D_peq_Ma_times_xD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_peq_Ma_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_meq_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_D_meq_M_times_xD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_meq_M_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_meq_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_D_meq_Ma_times_xD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_meq_Ma_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_eqm_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_D_eqm_M_times_xD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_eqm_M_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_eqm_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_D_eqm_Ma_times_xD");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_eqm_Ma_times_xD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_M_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_M_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_M_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_M_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_M_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_M_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_M_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_M_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_M_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_M_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_M_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_M_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_Ma_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_Ma_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_Ma_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_Ma_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_Ma_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_Ma_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_Ma_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_Ma_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_Ma_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_Ma_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_Ma_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_Ma_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_pM_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pM_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_pM_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_pM_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pM_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_pM_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_pM_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pM_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_pM_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_pM_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pM_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_pM_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_pMa_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pMa_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_pMa_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_pMa_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pMa_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_pMa_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_pMa_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pMa_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_pMa_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_pMa_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pMa_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_pMa_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_M_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_M_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_M_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_M_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_M_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_M_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_M_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_M_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_M_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_M_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_M_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_M_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_Ma_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_Ma_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_Ma_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_Ma_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_Ma_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_Ma_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_Ma_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_Ma_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_Ma_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_Ma_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_Ma_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_Ma_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_pM_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pM_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_pM_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_pM_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pM_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_pM_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_pM_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pM_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_pM_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_pM_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pM_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_pM_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_pMa_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pMa_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_pMa_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_pMa_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pMa_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_pMa_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_pMa_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pMa_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_pMa_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_pMa_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pMa_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_pMa_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_M_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_M_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_M_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_M_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_M_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_M_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_M_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_M_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_M_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_M_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_M_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_M_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_Ma_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_Ma_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_Ma_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_Ma_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_Ma_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_Ma_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_Ma_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_Ma_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_Ma_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_Ma_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_Ma_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_Ma_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_pM_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pM_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_pM_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_pM_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pM_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_pM_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_pM_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pM_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_pM_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_pM_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pM_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_pM_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_pMa_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pMa_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_pMa_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_pMa_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pMa_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_pMa_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_pMa_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pMa_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_pMa_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_pMa_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pMa_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_pMa_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_M_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_M_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_M_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_M_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_M_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_M_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_M_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_M_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_M_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_M_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_M_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_M_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_Ma_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_Ma_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_Ma_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_Ma_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_Ma_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_Ma_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_Ma_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_Ma_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_Ma_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_Ma_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_Ma_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_Ma_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_pM_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pM_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_pM_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_pM_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pM_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_pM_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_pM_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pM_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_pM_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_pM_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pM_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_pM_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_pMa_times_M(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pMa_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_pMa_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_pMa_times_pM(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pMa_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_pMa_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_pMa_times_Ma(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pMa_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_pMa_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_pMa_times_pMa(int nc, void * r, void * a, void * b, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pMa_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_pMa_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_M_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_M_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_M_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_M_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_M_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_M_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_M_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_M_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_M_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_M_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_M_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_M_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_Ma_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_Ma_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_Ma_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_Ma_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_Ma_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_Ma_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_Ma_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_Ma_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_Ma_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_Ma_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_Ma_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_Ma_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_pM_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pM_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_pM_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_pM_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pM_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_pM_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_pM_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pM_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_pM_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_pM_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pM_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_pM_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_pMa_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pMa_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_pMa_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_pMa_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pMa_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_pMa_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_pMa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pMa_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_pMa_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_pMa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pMa_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_pMa_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_M_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_M_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_M_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_M_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_M_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_M_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_M_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_M_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_M_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_M_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_M_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_M_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_Ma_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_Ma_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_Ma_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_Ma_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_Ma_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_Ma_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_Ma_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_Ma_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_Ma_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_Ma_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_Ma_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_Ma_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_pM_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pM_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_pM_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_pM_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pM_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_pM_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_pM_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pM_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_pM_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_pM_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pM_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_pM_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_pMa_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pMa_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_pMa_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_pMa_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pMa_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_pMa_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_pMa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pMa_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_pMa_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_pMa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pMa_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_pMa_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_M_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_M_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_M_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_M_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_M_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_M_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_M_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_M_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_M_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_M_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_M_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_M_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_Ma_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_Ma_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_Ma_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_Ma_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_Ma_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_Ma_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_Ma_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_Ma_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_Ma_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_Ma_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_Ma_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_Ma_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_pM_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pM_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_pM_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_pM_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pM_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_pM_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_pM_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pM_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_pM_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_pM_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pM_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_pM_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_pMa_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pMa_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_pMa_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_pMa_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pMa_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_pMa_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_pMa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pMa_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_pMa_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_pMa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pMa_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_pMa_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_M_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_M_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_M_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_M_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_M_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_M_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_M_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_M_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_M_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_M_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_M_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_M_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_Ma_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_Ma_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_Ma_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_Ma_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_Ma_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_Ma_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_Ma_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_Ma_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_Ma_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_Ma_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_Ma_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_Ma_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_pM_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pM_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_pM_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_pM_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pM_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_pM_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_pM_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pM_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_pM_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_pM_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pM_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_pM_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_pMa_times_M(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pMa_times_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_pMa_times_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_pMa_times_pM(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pMa_times_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_pMa_times_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_pMa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pMa_times_Ma");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_pMa_times_Ma", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_pMa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pMa_times_pMa");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, true>>("FN_lmult", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_pMa_times_pMa", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_eq_M_times_xM(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_M_eq_M_times_xM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_eq_M_times_xM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_eq_Ma_times_xM(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_M_eq_Ma_times_xM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_eq_Ma_times_xM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_peq_M_times_xM(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_M_peq_M_times_xM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_peq_M_times_xM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_peq_Ma_times_xM(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_M_peq_Ma_times_xM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_peq_Ma_times_xM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_meq_M_times_xM(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_M_meq_M_times_xM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_meq_M_times_xM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_meq_Ma_times_xM(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_M_meq_Ma_times_xM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_meq_Ma_times_xM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_eqm_M_times_xM(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_M_eqm_M_times_xM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, false, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_eqm_M_times_xM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_eqm_Ma_times_xM(int nc, void * r, void * a, void * b, int * jb, int n) {
  QLAB_TRACE("QLA_FN_M_eqm_Ma_times_xM");
  switch (nc) {
    case 2: qlab::api_map<qlab::LMultOp<float, 2, 2, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::LMultOp<float, 3, 3, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::LMultOp<float, 4, 4, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::LMultOp<float, 8, 8, true, false>>("FN_lmult", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_eqm_Ma_times_xM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

}  // extern "C"
