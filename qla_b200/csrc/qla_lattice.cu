// qla_lattice.cu -- device builder of periodic neighbour index streams.
//
// The reference receives neighbour gathers as arrays of pointers built by the
// caller (QDP's shift maps, doc/qla.tex:555-575).  On the GPU the natural
// form is an int32 index stream, built on the device once per (lattice, mu,
// sign) and passed to the `..._times_xV` / `..._eq_xV` entry points.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

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

// The first position of idx[0..n) whose entry lies outside [0, nsrc), and
// the number of such positions (both accumulated with atomics; first starts
// at ~0, count at 0).
__global__ void check_index_kernel(const int* __restrict__ idx, long long n, long long nsrc,
                                   unsigned long long* first, unsigned long long* count) {
  unsigned long long mine = ~0ull, c = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long v = __ldg(idx + i);
    if (v < 0 || v >= nsrc) {
      if (mine == ~0ull) mine = (unsigned long long)i;
      c++;
    }
  }
  for (int m = 16; m >= 1; m >>= 1) {
    const unsigned long long o = __shfl_xor_sync(0xffffffffu, mine, m);
    mine = o < mine ? o : mine;
    c += __shfl_xor_sync(0xffffffffu, c, m);
  }
  if ((threadIdx.x & 31) == 0 && c) {
    atomicMin(first, mine);
    atomicAdd(count, c);
  }
}

}  // namespace qlab

extern "C" QLAB_EXPORT int qlagpu_check_index(const int* idx, long long n, long long nsrc, long long* first_bad) {
  using namespace qlab;
  const char* who = "qlagpu_check_index";
  if (first_bad) *first_bad = -1;
  if (n < 0 || nsrc < 0) {
    set_error(QLAGPU_ERR_ARG, who, "n and nsrc must not be negative");
    return QLAGPU_ERR_ARG;
  }
  if (n == 0) return QLAGPU_OK;
  if (!idx) {
    set_error(QLAGPU_ERR_NULLPTR, who, "NULL index stream");
    return QLAGPU_ERR_NULLPTR;
  }
  // two 8-B words per device, allocated on the first call
  static std::mutex mu;
  static unsigned long long* words[64] = {nullptr};
  const int dev = current_device();
  if (dev < 0 || dev >= 64) {
    set_error(QLAGPU_ERR_ARG, who, "device ordinal out of range");
    return QLAGPU_ERR_ARG;
  }
  unsigned long long* w;
  {
    std::lock_guard<std::mutex> g(mu);
    if (!words[dev] && cudaMalloc(&words[dev], 2 * sizeof(unsigned long long)) != cudaSuccess) {
      words[dev] = nullptr;
      cudaGetLastError();
      set_error(QLAGPU_ERR_ALLOC, who, "cudaMalloc failed");
      return QLAGPU_ERR_ALLOC;
    }
    w = words[dev];
  }
  cudaStream_t st = current_stream();
  unsigned long long host[2] = {~0ull, 0ull};
  const int threads = 256;
  long long blocks = (n + threads - 1) / threads;
  const long long cap = (long long)device_sm_count() * 8;
  if (blocks > cap) blocks = cap;
  if (cudaMemcpyAsync(w, host, sizeof(host), cudaMemcpyHostToDevice, st) != cudaSuccess) {
    check_launch(who);
    return QLAGPU_ERR_LAUNCH;
  }
  check_index_kernel<<<(unsigned)blocks, threads, 0, st>>>(idx, n, nsrc, w, w + 1);
  if (!check_launch(who) || cudaMemcpyAsync(host, w, sizeof(host), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    check_launch(who);
    return QLAGPU_ERR_LAUNCH;
  }
  if (host[1] == 0) return QLAGPU_OK;
  int v = 0;
  cudaMemcpy(&v, idx + host[0], sizeof(int), cudaMemcpyDeviceToHost);
  if (first_bad) *first_bad = (long long)host[0];
  char msg[160];
  std::snprintf(msg, sizeof msg, "%llu entries outside [0, %lld); the first at position %llu holds %d", host[1], nsrc,
                host[0], v);
  set_error(QLAGPU_ERR_ARG, who, msg);
  return QLAGPU_ERR_ARG;
}

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
