// qla_lattice.cu -- device builder of periodic neighbour index streams.
//
// The reference receives neighbour gathers as arrays of pointers built by the
// caller (QDP's shift maps, doc/qla.tex:555-575).  On the GPU the natural
// form is an int32 index stream, built on the device once per (lattice, mu,
// sign) and passed to the `..._times_xV` / `..._eq_xV` entry points.
#include <cuda_runtime.h>

#include "../../include/qla_b200_runtime.h"
#include "qla_runtime.h"

namespace qlab {

struct Dims {
  int nd;
  int L[8];
};

// idx[i] = lexicographic index (x0 fastest) of coord(i) + sign * e_mu, periodic
__global__ void shift_index_kernel(int* __restrict__ idx, Dims d, int mu, int sign, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    long long rem = i, stride = 1, out = 0;
    for (int k = 0; k < d.nd; k++) {
      const int L = d.L[k];
      long long c = rem % L;
      rem /= L;
      if (k == mu) {
        c += sign;
        if (c < 0) c += L;
        if (c >= L) c -= L;
      }
      out += c * stride;
      stride *= L;
    }
    idx[i] = (int)out;
  }
}

}  // namespace qlab

extern "C" QLAB_EXPORT void qlagpu_shift_index(int* idx, int nd, const int* dims, int mu, int sign) {
  using namespace qlab;
  if (!idx || !dims) {
    set_error(QLAGPU_ERR_NULLPTR, "qlagpu_shift_index", "NULL argument");
    return;
  }
  if (nd < 1 || nd > 8 || mu < 0 || mu >= nd || (sign != 1 && sign != -1)) {
    set_error(QLAGPU_ERR_ARG, "qlagpu_shift_index", "need 1<=nd<=8, 0<=mu<nd, sign=+-1");
    return;
  }
  Dims d;
  d.nd = nd;
  long long n = 1;
  for (int k = 0; k < nd; k++) {
    if (dims[k] < 1) {
      set_error(QLAGPU_ERR_ARG, "qlagpu_shift_index", "extent < 1");
      return;
    }
    d.L[k] = dims[k];
    n *= dims[k];
  }
  if (n > 0x7fffffffLL) {
    set_error(QLAGPU_ERR_ARG, "qlagpu_shift_index", "volume exceeds int32");
    return;
  }
  const int threads = 256;
  long long blocks = (n + threads - 1) / threads;
  const long long cap = (long long)device_sm_count() * 16;
  if (blocks > cap) blocks = cap;
  shift_index_kernel<<<(unsigned)blocks, threads, 0, current_stream()>>>(idx, d, mu, sign, n);
  check_launch("qlagpu_shift_index");
}
