// qla_int.cuh -- QLA_I_ integer site operations (lib/perl/build_qla.pl:1932-2082):
// r[i] (eqop) f(a[i], b[i], c[i], *s) on int32 fields, bit-exact with the
// reference's C semantics (two's-complement wrap on overflow, `/` and `%`
// truncate toward zero, `>>` arithmetic, comparisons give 0/1, mask keeps r
// where the mask is zero).  Inputs the reference leaves undefined (b == 0,
// INT_MIN / -1, shift counts outside 0..31) stay undefined here.
//
// HBM-bound streaming: one kernel, four sites per thread with 16-B vector
// accesses when every contiguous operand is 16-B aligned and no gang index is
// used, one site per thread otherwise.
#pragma once
#include "qla_engine.cuh"
#include "qla_launch.cuh"

namespace qlab {

enum IntCode : int {
  IC_COPY = 0, IC_TIMES, IC_PLUS, IC_MINUS, IC_DIVIDE, IC_MOD, IC_AND, IC_OR, IC_XOR, IC_LSHIFT, IC_RSHIFT,
  IC_EQ, IC_NE, IC_LT, IC_LE, IC_GT, IC_GE, IC_MAX, IC_MIN, IC_MASK, IC_NOT, IC_ZERO,
  IC_S, IC_S_TIMES, IC_S_TIMES_PLUS, IC_S_TIMES_MINUS
};

struct IntParams {
  Opnd in[3];
  int* out;
  const int* gang;
  const int* sptr;  // scalar on the device
  int sval;         // scalar read on the host
  int code, eqop, nin, vec;
  long long n;
};

__device__ __forceinline__ int int_value(int code, int a, int b, int c, int s) {
  switch (code) {
    case IC_COPY: return a;
    case IC_TIMES: return (int)((unsigned)a * (unsigned)b);
    case IC_PLUS: return (int)((unsigned)a + (unsigned)b);
    case IC_MINUS: return (int)((unsigned)a - (unsigned)b);
    case IC_DIVIDE: return a / b;
    case IC_MOD: return a % b;
    case IC_AND: return a & b;
    case IC_OR: return a | b;
    case IC_XOR: return a ^ b;
    case IC_LSHIFT: return (int)((unsigned)a << b);
    case IC_RSHIFT: return a >> b;
    case IC_EQ: return a == b;
    case IC_NE: return a != b;
    case IC_LT: return a < b;
    case IC_LE: return a <= b;
    case IC_GT: return a > b;
    case IC_GE: return a >= b;
    case IC_MAX: return a > b ? a : b;
    case IC_MIN: return a < b ? a : b;
    case IC_NOT: return !a;
    case IC_ZERO: return 0;
    case IC_S: return s;
    case IC_S_TIMES: return (int)((unsigned)s * (unsigned)a);
    case IC_S_TIMES_PLUS: return (int)((unsigned)s * (unsigned)a + (unsigned)b);
    default: return (int)((unsigned)s * (unsigned)a - (unsigned)b);  // IC_S_TIMES_MINUS
  }
}

// r (eqop) v ; mask: r = a where b != 0
__device__ __forceinline__ int int_apply(int code, int eqop, int r, int a, int b, int c, int s) {
  if (code == IC_MASK) return b ? a : r;
  const int v = int_value(code, a, b, c, s);
  switch (eqop) {
    case EQ: return v;
    case PEQ: return (int)((unsigned)r + (unsigned)v);
    case MEQ: return (int)((unsigned)r - (unsigned)v);
    default: return (int)(0u - (unsigned)v);
  }
}

__device__ __forceinline__ int int_fetch(const Opnd& o, long long k) {
  if (o.mode == OM_PTR) return *static_cast<const int*>(o.ptrs[k]);
  if (o.mode == OM_IDX) return static_cast<const int*>(o.base)[o.idx[k]];
  return static_cast<const int*>(o.base)[k];
}

__global__ void __launch_bounds__(256) int_kernel(const IntParams p) {
  const int s = p.sptr ? __ldg(p.sptr) : p.sval;
  const bool rd = (p.eqop == PEQ || p.eqop == MEQ || p.code == IC_MASK);
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (p.vec) {
    // four sites per thread, 16-B accesses on contiguous operands
    const long long n4 = p.n / 4;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += stride) {
      int4 av = make_int4(0, 0, 0, 0), bv = av, cv = av, rv = av;
      if (p.nin > 0) av = __ldg(static_cast<const int4*>(p.in[0].base) + q);
      if (p.nin > 1) bv = __ldg(static_cast<const int4*>(p.in[1].base) + q);
      if (p.nin > 2) cv = __ldg(static_cast<const int4*>(p.in[2].base) + q);
      if (rd) rv = reinterpret_cast<const int4*>(p.out)[q];
      rv.x = int_apply(p.code, p.eqop, rv.x, av.x, bv.x, cv.x, s);
      rv.y = int_apply(p.code, p.eqop, rv.y, av.y, bv.y, cv.y, s);
      rv.z = int_apply(p.code, p.eqop, rv.z, av.z, bv.z, cv.z, s);
      rv.w = int_apply(p.code, p.eqop, rv.w, av.w, bv.w, cv.w, s);
      reinterpret_cast<int4*>(p.out)[q] = rv;
    }
    for (long long k = n4 * 4 + (long long)blockIdx.x * blockDim.x + threadIdx.x; k < p.n; k += stride) {
      const int a = p.nin > 0 ? int_fetch(p.in[0], k) : 0;
      const int b = p.nin > 1 ? int_fetch(p.in[1], k) : 0;
      const int c = p.nin > 2 ? int_fetch(p.in[2], k) : 0;
      p.out[k] = int_apply(p.code, p.eqop, rd ? p.out[k] : 0, a, b, c, s);
    }
    return;
  }
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += stride) {
    const long long k = p.gang ? (long long)p.gang[i] : i;
    const int a = p.nin > 0 ? int_fetch(p.in[0], k) : 0;
    const int b = p.nin > 1 ? int_fetch(p.in[1], k) : 0;
    const int c = p.nin > 2 ? int_fetch(p.in[2], k) : 0;
    p.out[k] = int_apply(p.code, p.eqop, rd ? p.out[k] : 0, a, b, c, s);
  }
}

// host entry for the generated QLA_I_ wrappers
inline void api_int(const char* kid, int code, int eqop, int* r, const int* s, Opnd a, Opnd b, Opnd c, int nin,
                    const int* gang, int n) {
  if (n <= 0) return;
  const Opnd ops[3] = {a, b, c};
  bool bad = (r == nullptr) || ((code == IC_S || code >= IC_S_TIMES) && s == nullptr);
  for (int j = 0; j < nin; j++)
    if ((ops[j].mode == OM_CONTIG && !ops[j].base) || (ops[j].mode == OM_PTR && !ops[j].ptrs)) bad = true;
  if (bad) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  IntParams p;
  std::memset(&p, 0, sizeof(p));
  p.in[0] = a;
  p.in[1] = b;
  p.in[2] = c;
  p.out = r;
  p.gang = gang;
  p.code = code;
  p.eqop = eqop;
  p.nin = nin;
  p.n = n;
  if (s) {
    if (is_device_ptr(s))
      p.sptr = s;
    else
      p.sval = *s;
  }
  bool vec = (gang == nullptr) && aligned16(r);
  for (int j = 0; j < nin; j++) vec = vec && ops[j].mode == OM_CONTIG && aligned16(ops[j].base);
  p.vec = vec ? 1 : 0;
  const int threads = 256;
  long long want = ((vec ? (long long)n / 4 : (long long)n) + threads - 1) / threads;
  const long long cap = (long long)device_sm_count() * 16;
  if (want > cap) want = cap;
  if (want < 1) want = 1;
  int_kernel<<<(unsigned)want, threads, 0, current_stream()>>>(p);
  check_launch(kid);
}

}  // namespace qlab
