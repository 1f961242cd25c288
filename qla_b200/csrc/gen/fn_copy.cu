// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA FN copy entry points (extern "C"), reference: lib/perl/build_qla.pl:370-400 (assignment / gather)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_FN_V_veq_V(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_V_veq_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 2>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 3>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veq_pV(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_V_veq_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 2>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 3>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veq_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vpeq_V(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_V_vpeq_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 2>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 3>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vpeq_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vpeq_pV(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_V_vpeq_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 2>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 3>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vpeq_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vmeq_V(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_V_vmeq_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 2>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 3>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vmeq_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_vmeq_pV(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_V_vmeq_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 2>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 3>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_vmeq_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veqm_V(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_V_veqm_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 2>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 3>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veqm_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_veqm_pV(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_V_veqm_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 2>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 3>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_veqm_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_V(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 2>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 3>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeq_pV(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeq_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 2>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 3>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeq_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xpeq_V(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xpeq_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 2>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 3>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xpeq_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xpeq_pV(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xpeq_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 2>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 3>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xpeq_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xmeq_V(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xmeq_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 2>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 3>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xmeq_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xmeq_pV(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xmeq_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 2>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 3>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xmeq_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeqm_V(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeqm_V");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 2>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 3>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeqm_V", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_V_xeqm_pV(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_V_xeqm_pV");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 2>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 3>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_V_xeqm_pV", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veq_H(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_H_veq_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 6>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veq_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veq_pH(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_H_veq_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 6>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veq_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vpeq_H(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_H_vpeq_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 6>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vpeq_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vpeq_pH(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_H_vpeq_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 6>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vpeq_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vmeq_H(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_H_vmeq_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 6>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vmeq_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_vmeq_pH(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_H_vmeq_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 6>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_vmeq_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veqm_H(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_H_veqm_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 6>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veqm_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_veqm_pH(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_H_veqm_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 6>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_veqm_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeq_H(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeq_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 6>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeq_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeq_pH(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeq_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 6>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeq_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xpeq_H(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xpeq_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 6>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xpeq_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xpeq_pH(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xpeq_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 6>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xpeq_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xmeq_H(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xmeq_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 6>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xmeq_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xmeq_pH(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xmeq_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 6>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xmeq_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeqm_H(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeqm_H");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 6>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeqm_H", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_H_xeqm_pH(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_H_xeqm_pH");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 6>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_H_xeqm_pH", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veq_D(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_D_veq_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 12>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 32>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veq_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veq_pD(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_D_veq_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 12>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 32>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veq_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vpeq_D(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_D_vpeq_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 12>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 32>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vpeq_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vpeq_pD(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_D_vpeq_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 12>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 32>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vpeq_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vmeq_D(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_D_vmeq_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 12>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 32>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vmeq_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_vmeq_pD(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_D_vmeq_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 12>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 32>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_vmeq_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veqm_D(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_D_veqm_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 12>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 32>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veqm_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_veqm_pD(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_D_veqm_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 12>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 32>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_veqm_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeq_D(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeq_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 12>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 32>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeq_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeq_pD(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeq_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 12>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 32>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeq_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xpeq_D(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xpeq_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 12>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 32>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xpeq_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xpeq_pD(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xpeq_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 12>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 32>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xpeq_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xmeq_D(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xmeq_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 12>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 32>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xmeq_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xmeq_pD(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xmeq_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 12>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 32>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xmeq_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeqm_D(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeqm_D");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 12>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 32>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeqm_D", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_D_xeqm_pD(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_D_xeqm_pD");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 8>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 12>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 32>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_D_xeqm_pD", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 9>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 64>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veq_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veq_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 9>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 64>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veq_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 9>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 64>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vpeq_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vpeq_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 9>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 64>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vpeq_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 9>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 64>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_vmeq_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_vmeq_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 9>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 64>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_vmeq_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_M(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 9>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 64>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_veqm_pM(int nc, void * r, void * a, int n) {
  QLAB_TRACE("QLA_FN_M_veqm_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 9>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 64>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_veqm_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 9>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 64>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeq_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeq_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 9>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 64>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeq_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 9>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 64>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xpeq_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xpeq_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 9>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 64>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xpeq_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 9>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 64>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xmeq_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xmeq_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 9>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 64>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xmeq_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_M(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_M");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 9>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 64>>("FN_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_M", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

QLAB_EXPORT void QLA_FN_M_xeqm_pM(int nc, void * r, void * a, int * index, int n) {
  QLAB_TRACE("QLA_FN_M_xeqm_pM");
  switch (nc) {
    case 2: qlab::api_map<qlab::CopyOp<float, 4>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 3: qlab::api_map<qlab::CopyOp<float, 9>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 4: qlab::api_map<qlab::CopyOp<float, 16>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM); break;
    case 8: qlab::api_map<qlab::CopyOp<float, 64>>("FN_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM); break;
    default: qlab::set_error(QLAGPU_ERR_ARG, "QLA_FN_M_xeqm_pM", "nc not compiled (supported: 2, 3, 4, 8)");
  }
}

}  // extern "C"
