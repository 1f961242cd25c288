// qla_scalar.cuh -- the real- and complex-field libraries QLA_F_ / QLA_D_
// (one real, complex or integer number per site) and the DF / FD precision
// conversions and double-precision reductions of QLA_DF_.
//
// Complex-field products, sums, constant multiples, conj / i copies, fills,
// masks and the site-local dot products run on the element-wise kernels of
// qla_ewise.cuh / qla_sitefield.cuh with a record of one complex number.
// This file adds what those do not cover: real- and integer-valued fields
// (copies and eqop updates, arithmetic, comparisons, rounding, the libm
// functions), the complex functions of lib/cmath (cexp, cexpi, clog, csqrt),
// complex division, the complex <-> real conversions, the global reductions
// and sums of real / integer fields, and real precision conversions.
//
// Reference: lib/perl/build_qla.pl:186-355 (elementary functions, real /
// complex conversions), :1936-2082 (comparisons, rounding, masks),
// :2089-2555 (global reductions and sums); include/qla_complex.h:110-140,
// 417-428 (norm, arg, division); lib/cmath/QLA_cexp.c, QLA_cexpi.c,
// QLA_clog.c, QLA_csqrt.c.
//
// Exactness: every operation built from + - * / sqrt, comparisons,
// conversions, fabs / ceil / floor / round / trunc, fmod and ldexp is
// bit-identical to the reference.  The transcendental functions (sin ... tanh,
// exp, log, pow, atan2 and the cmath functions built on them) use CUDA's
// implementations, which agree with the host libm to within a few units in
// the last place; the F library's pow / atan2 / log are evaluated in double
// and rounded to float as the reference does, so they almost always agree
// exactly.
#pragma once
#include <type_traits>
#include "qla_sitefield.cuh"

namespace qlab {

enum ScalarOp : int {
  // real result, any eqop
  SO_R_COPY = 0,    // r (eqop) a
  SO_R_TIMES_R,     // r (eqop) a * b
  SO_R_RTIMES,      // r (eqop) s * b            (s a real constant)
  SO_R_FILL,        // r (eqop) s
  // real result, eq only
  SO_R_ZERO,
  SO_R_MASK,        // if (b) r = a
  SO_R_FROM_I,      // r = (real) a
  SO_R_PLUS, SO_R_MINUS, SO_R_DIVIDE, SO_R_MAX, SO_R_MIN,
  SO_R_MOD,         // fmod(a, b)
  SO_R_POW,         // pow(a, b)
  SO_R_ATAN2,       // atan2(a, b)
  SO_R_LDEXP,       // ldexp(a, b), b an integer field
  SO_R_RT_PLUS,     // s * b + c
  SO_R_RT_MINUS,    // s * b - c
  SO_R_SIN, SO_R_COS, SO_R_TAN, SO_R_ASIN, SO_R_ACOS, SO_R_ATAN, SO_R_SQRT, SO_R_FABS, SO_R_EXP,
  SO_R_LOG, SO_R_LOG10, SO_R_SINH, SO_R_COSH, SO_R_TANH, SO_R_CEIL, SO_R_FLOOR, SO_R_SIGN,
  SO_R_RE,          // Re a (a complex)
  SO_R_IM,          // Im a
  SO_R_NORM,        // |a|
  SO_R_ARG,         // arg a
  // integer result
  SO_I_EQ, SO_I_GE, SO_I_GT, SO_I_LE, SO_I_LT, SO_I_NE,   // a (op) b
  SO_I_ROUND, SO_I_TRUNC,
  // complex result
  SO_C_FROM_R,      // a + 0 i
  SO_C_R_PLUS_I_R,  // a + i b
  SO_C_DIVIDE,      // a / b
  SO_C_CEXP, SO_C_CEXPI, SO_C_CLOG, SO_C_CSQRT
};

struct ScParams {
  void* out;
  Opnd a, b, c;
  const int* gang;
  long long n;
  int eqop;
  double sre;          // real constant passed by value
  const void* sptr;    // real constant left on the device
};

template <typename T>
__device__ __forceinline__ T ld_s(const Opnd& o, long long k) {
  return (o.mode == OM_PTR) ? *static_cast<const T*>(o.ptrs[k]) : static_cast<const T*>(o.base)[k];
}

// libm functions in the library's precision (the F library calls the float
// functions, the D library the double ones)
template <typename R>
__device__ __forceinline__ R math1(int op, R x) {
  if constexpr (sizeof(R) == 4) {
    switch (op) {
      case SO_R_SIN: return sinf(x);
      case SO_R_COS: return cosf(x);
      case SO_R_TAN: return tanf(x);
      case SO_R_ASIN: return asinf(x);
      case SO_R_ACOS: return acosf(x);
      case SO_R_ATAN: return atanf(x);
      case SO_R_SQRT: return __fsqrt_rn(x);
      case SO_R_FABS: return fabsf(x);
      case SO_R_EXP: return expf(x);
      case SO_R_LOG: return logf(x);
      case SO_R_LOG10: return log10f(x);
      case SO_R_SINH: return sinhf(x);
      case SO_R_COSH: return coshf(x);
      case SO_R_TANH: return tanhf(x);
      case SO_R_CEIL: return ceilf(x);
      default: return floorf(x);
    }
  } else {
    switch (op) {
      case SO_R_SIN: return sin(x);
      case SO_R_COS: return cos(x);
      case SO_R_TAN: return tan(x);
      case SO_R_ASIN: return asin(x);
      case SO_R_ACOS: return acos(x);
      case SO_R_ATAN: return atan(x);
      case SO_R_SQRT: return __dsqrt_rn(x);
      case SO_R_FABS: return fabs(x);
      case SO_R_EXP: return exp(x);
      case SO_R_LOG: return log(x);
      case SO_R_LOG10: return log10(x);
      case SO_R_SINH: return sinh(x);
      case SO_R_COSH: return cosh(x);
      case SO_R_TANH: return tanh(x);
      case SO_R_CEIL: return ceil(x);
      default: return floor(x);
    }
  }
}

template <typename R>
__device__ __forceinline__ R norm2_r(Cx<R> a) {
  return radd(rmul(a.re, a.re), rmul(a.im, a.im));
}

template <typename R>
__device__ __forceinline__ R sqrt_r(R x) {
  if constexpr (sizeof(R) == 4)
    return __fsqrt_rn(x);
  else
    return __dsqrt_rn(x);
}

template <typename R>
__device__ __forceinline__ R atan2_r(R y, R x) {
  if constexpr (sizeof(R) == 4)
    return atan2f(y, x);
  else
    return atan2(y, x);
}

template <typename R>
__device__ __forceinline__ void sincos_r(R x, R* s, R* c) {
  if constexpr (sizeof(R) == 4)
    sincosf(x, s, c);
  else
    sincos(x, s, c);
}

// the eqop update of a real result (r = t, r += t, r -= t, r = -t)
template <typename R>
__device__ __forceinline__ R r_eqop(int eqop, R x, R t) {
  switch (eqop) {
    case EQ: return t;
    case PEQ: return radd(x, t);
    case MEQ: return rsub(x, t);
    default: return -t;
  }
}

template <typename R, int OP>
__global__ void __launch_bounds__(256) scalar_kernel(const ScParams p) {
  R sv = R(0);
  if constexpr (OP == SO_R_RTIMES || OP == SO_R_FILL || OP == SO_R_RT_PLUS || OP == SO_R_RT_MINUS)
    sv = p.sptr ? *static_cast<const R*>(p.sptr) : (R)p.sre;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < p.n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long k = p.gang ? (long long)p.gang[i] : i;
    if constexpr (OP <= SO_R_ARG) {
      R* out = static_cast<R*>(p.out) + k;
      if constexpr (OP == SO_R_COPY) {
        *out = r_eqop<R>(p.eqop, (p.eqop == PEQ || p.eqop == MEQ) ? *out : R(0), ld_s<R>(p.a, k));
      } else if constexpr (OP == SO_R_TIMES_R) {
        const R a = ld_s<R>(p.a, k), b = ld_s<R>(p.b, k);
        // eqm: r = -a * b, the same value as -(a * b)
        *out = r_eqop<R>(p.eqop, (p.eqop == PEQ || p.eqop == MEQ) ? *out : R(0), rmul(a, b));
      } else if constexpr (OP == SO_R_RTIMES) {
        *out = r_eqop<R>(p.eqop, (p.eqop == PEQ || p.eqop == MEQ) ? *out : R(0), rmul(sv, ld_s<R>(p.b, k)));
      } else if constexpr (OP == SO_R_FILL) {
        *out = r_eqop<R>(p.eqop, (p.eqop == PEQ || p.eqop == MEQ) ? *out : R(0), sv);
      } else if constexpr (OP == SO_R_ZERO) {
        *out = R(0);
      } else if constexpr (OP == SO_R_MASK) {
        if (ld_s<int>(p.b, k)) *out = ld_s<R>(p.a, k);
      } else if constexpr (OP == SO_R_FROM_I) {
        *out = (R)ld_s<int>(p.a, k);
      } else if constexpr (OP == SO_R_LDEXP) {
        *out = (R)ldexp((double)ld_s<R>(p.a, k), ld_s<int>(p.b, k));
      } else if constexpr (OP >= SO_R_PLUS && OP <= SO_R_ATAN2) {
        const R a = ld_s<R>(p.a, k), b = ld_s<R>(p.b, k);
        R t;
        if constexpr (OP == SO_R_PLUS)
          t = radd(a, b);
        else if constexpr (OP == SO_R_MINUS)
          t = rsub(a, b);
        else if constexpr (OP == SO_R_DIVIDE)
          t = rdiv(a, b);
        else if constexpr (OP == SO_R_MAX)
          t = (a > b ? a : b);
        else if constexpr (OP == SO_R_MIN)
          t = (a > b ? b : a);
        else if constexpr (OP == SO_R_MOD)
          t = (R)fmod((double)a, (double)b);
        else if constexpr (OP == SO_R_POW)
          t = (R)pow((double)a, (double)b);
        else
          t = (R)atan2((double)a, (double)b);
        *out = t;
      } else if constexpr (OP == SO_R_RT_PLUS || OP == SO_R_RT_MINUS) {
        const R t = rmul(sv, ld_s<R>(p.b, k)), c = ld_s<R>(p.c, k);
        *out = (OP == SO_R_RT_PLUS) ? radd(t, c) : rsub(t, c);
      } else if constexpr (OP == SO_R_SIGN) {
        *out = ld_s<R>(p.a, k) >= R(0) ? R(1) : R(-1);
      } else if constexpr (OP >= SO_R_SIN && OP <= SO_R_FLOOR) {
        *out = math1<R>(OP, ld_s<R>(p.a, k));
      } else {
        const Cx<R> a = *rec_ptr<R>(p.a, k, 1);
        if constexpr (OP == SO_R_RE)
          *out = a.re;
        else if constexpr (OP == SO_R_IM)
          *out = a.im;
        else if constexpr (OP == SO_R_NORM)
          *out = sqrt_r<R>(norm2_r<R>(a));
        else
          *out = atan2_r<R>(a.im, a.re);
      }
    } else if constexpr (OP <= SO_I_TRUNC) {
      int* out = static_cast<int*>(p.out) + k;
      const R a = ld_s<R>(p.a, k);
      if constexpr (OP == SO_I_ROUND) {
        if constexpr (sizeof(R) == 4)
          *out = (int)roundf(a);
        else
          *out = (int)round(a);
      } else if constexpr (OP == SO_I_TRUNC) {
        *out = (int)a;
      } else {
        const R b = ld_s<R>(p.b, k);
        int t;
        if constexpr (OP == SO_I_EQ) t = (a == b);
        else if constexpr (OP == SO_I_GE) t = (a >= b);
        else if constexpr (OP == SO_I_GT) t = (a > b);
        else if constexpr (OP == SO_I_LE) t = (a <= b);
        else if constexpr (OP == SO_I_LT) t = (a < b);
        else t = (a != b);
        *out = t;
      }
    } else {
      Cx<R>* out = static_cast<Cx<R>*>(p.out) + k;
      if constexpr (OP == SO_C_FROM_R) {
        *out = Cx<R>{ld_s<R>(p.a, k), R(0)};
      } else if constexpr (OP == SO_C_R_PLUS_I_R) {
        *out = Cx<R>{ld_s<R>(p.a, k), ld_s<R>(p.b, k)};
      } else if constexpr (OP == SO_C_DIVIDE) {
        // t = 1.0 / |b|^2 (a double quotient stored in the site precision),
        // then (a conj(b)) t (include/qla_complex.h:417-427)
        const Cx<R> a = *rec_ptr<R>(p.a, k, 1), b = *rec_ptr<R>(p.b, k, 1);
        const R t = (R)__ddiv_rn(1.0, (double)norm2_r<R>(b));
        *out = Cx<R>{rmul(radd(rmul(a.re, b.re), rmul(a.im, b.im)), t),
                     rmul(rsub(rmul(a.im, b.re), rmul(a.re, b.im)), t)};
      } else if constexpr (OP == SO_C_CEXPI) {
        R s, c;
        sincos_r<R>(ld_s<R>(p.a, k), &s, &c);
        *out = Cx<R>{c, s};
      } else {
        const Cx<R> a = *rec_ptr<R>(p.a, k, 1);
        if constexpr (OP == SO_C_CEXP) {
          R s, c;
          R mag;
          if constexpr (sizeof(R) == 4)
            mag = expf(a.re);
          else
            mag = exp(a.re);
          sincos_r<R>(a.im, &s, &c);
          *out = Cx<R>{rmul(mag, c), rmul(mag, s)};
        } else if constexpr (OP == SO_C_CLOG) {
          // 0.5 * log(|a|^2) in double, the argument in the site precision
          *out = Cx<R>{(R)__dmul_rn(0.5, log((double)norm2_r<R>(a))), atan2_r<R>(a.im, a.re)};
        } else {
          // n = |a|; sqrt(|0.5 (n + re)|) + i copysign(sqrt(|0.5 (n - re)|), im),
          // the halving in double as the reference writes it
          const R n = sqrt_r<R>(norm2_r<R>(a));
          const R h1 = (R)__dmul_rn(0.5, (double)radd(n, a.re));
          const R h2 = (R)__dmul_rn(0.5, (double)rsub(n, a.re));
          const R si = sqrt_r<R>(h2 < R(0) ? -h2 : h2);
          R sg;
          if constexpr (sizeof(R) == 4)
            sg = copysignf(si, a.im);
          else
            sg = copysign(si, a.im);
          *out = Cx<R>{sqrt_r<R>(h1 < R(0) ? -h1 : h1), sg};
        }
      }
    }
  }
}

// r (eqop) op(a, b, c, s): s a real constant in host or device memory
template <typename R, int OP>
inline void api_scalar(const char* kid, void* r, const void* scal, Opnd a, Opnd b, Opnd c, const int* gang, int n,
                       int eqop) {
  if (n <= 0) return;
  constexpr bool SCAL = OP == SO_R_RTIMES || OP == SO_R_FILL || OP == SO_R_RT_PLUS || OP == SO_R_RT_MINUS;
  if (!r || !opnd_ok(a) || !opnd_ok(b) || !opnd_ok(c) || (SCAL && !scal)) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  ScParams p;
  std::memset(&p, 0, sizeof(p));
  p.out = r;
  p.a = a;
  p.b = b;
  p.c = c;
  p.gang = gang;
  p.n = n;
  p.eqop = eqop;
  if constexpr (SCAL) {
    if (is_device_ptr(scal))
      p.sptr = scal;
    else
      p.sre = (double)*static_cast<const R*>(scal);
  }
  const long long cap = (long long)device_sm_count() * 16;
  long long grid = ((long long)n + 255) / 256;
  if (grid > cap) grid = cap;
  scalar_kernel<R, OP><<<(unsigned)(grid < 1 ? 1 : grid), 256, 0, current_stream()>>>(p);
  check_launch(kid);
}

// ---------------------------------------------------------------------------
// global reductions of real / integer fields: each site's term is formed as
// the reference forms it (the product or square in the field's arithmetic:
// float for QLA_F_ and QLA_DF_ on float fields, int for integer products),
// the sites are added in double-double (build_qla.pl:2089-2555)
enum SredKind : int { SR_DOT = 0, SR_NORM2 = 1, SR_SUM = 2 };

template <int NACC_, typename OUT>
struct SredFinish {
  static constexpr int NACC = NACC_;
  __device__ static void finish(const SiteParams& p, const double* tot) { write_real<OUT>(p, tot[0]); }
};

// RIN: field element type (float, double or int); RW: the library's real type
// Eight terms in flight per thread, summed in double by tree_sum (exact for
// integer fields below 2^53), each group added in double-double.
template <typename RIN, typename RW, int KIND, typename OUT>
__global__ void __launch_bounds__(256) sred_kernel(const EwParams p, const SiteParams rp) {
  constexpr int U = 8;
  DD acc[1] = {DD{0.0, 0.0}};
  auto term = [&](long long i) -> double {
    const long long k = p.gang ? (long long)p.gang[i] : i;
    const RIN a = ld_s<RIN>(p.b, k);
    if constexpr (KIND == SR_SUM) {
      return (double)a;
    } else if constexpr (KIND == SR_DOT) {
      const RIN b = ld_s<RIN>(p.c, k);
      if constexpr (std::is_same<RIN, int>::value)  // the product wraps as the reference's int product
        return (double)(int)((unsigned)a * (unsigned)b);
      else
        return (double)rmul(a, b);
    } else {
      const RW at = (RW)a;
      return (double)rmul(at, at);
    }
  };
  const long long stride = (long long)gridDim.x * blockDim.x;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + (U - 1) * stride < p.n; i += U * stride) {
    double t[U];
#pragma unroll
    for (int u = 0; u < U; u++) t[u] = term(i + u * stride);
    dd_add(acc[0], tree_sum(t));
  }
  for (; i < p.n; i += stride) dd_add(acc[0], term(i));
  reduce_finish<SredFinish<1, OUT>>(rp, acc);
}

template <typename RIN, typename RW, int KIND, typename OUT>
inline void api_sred(const char* kid, void* r, Opnd a, Opnd b, const int* gang, int n) {
  const size_t rbytes = sizeof(OUT);
  if (!r || (n > 0 && (!opnd_ok(a) || (KIND == SR_DOT && !opnd_ok(b))))) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  cudaStream_t st = current_stream();
  const bool dev_out = is_device_ptr(r);
  if (n <= 0) {
    if (dev_out)
      cudaMemsetAsync(r, 0, rbytes, st);
    else
      std::memset(r, 0, rbytes);
    return;
  }
  const int sms = device_sm_count();
  ReduceScratch* rs = reduce_scratch(st, 32 * sms + 64);
  if (!rs) return;
  EwParams p;
  std::memset(&p, 0, sizeof(p));
  p.b = a;
  p.c = b;
  p.gang = gang;
  p.n = n;
  SiteParams rp;
  std::memset(&rp, 0, sizeof(rp));
  rp.partials = rs->partials;
  rp.counter = rs->counter;
  rp.result = dev_out ? r : rs->result;
  long long grid = ((long long)n + 255) / 256;
  const long long cap = (long long)sms * 4;
  if (grid > cap) grid = cap;
  if (grid > rs->max_blocks) grid = rs->max_blocks;
  sred_kernel<RIN, RW, KIND, OUT><<<(unsigned)(grid < 1 ? 1 : grid), 256, 0, st>>>(p, rp);
  if (!check_launch(kid)) return;
  if (!dev_out) {
    if (cudaMemcpyAsync(r, rs->result, rbytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      check_launch(kid);
  }
}

// real precision conversion r = (ROUT) a
template <typename RIN, typename ROUT>
__global__ void __launch_bounds__(256) rconvert_kernel(const ScParams p) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < p.n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long k = p.gang ? (long long)p.gang[i] : i;
    static_cast<ROUT*>(p.out)[k] = static_cast<ROUT>(ld_s<RIN>(p.a, k));
  }
}

template <typename RIN, typename ROUT>
inline void api_rconvert(const char* kid, void* r, Opnd a, const int* gang, int n) {
  if (n <= 0) return;
  if (!r || !opnd_ok(a)) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  ScParams p;
  std::memset(&p, 0, sizeof(p));
  p.out = r;
  p.a = a;
  p.gang = gang;
  p.n = n;
  const long long cap = (long long)device_sm_count() * 16;
  long long grid = ((long long)n + 255) / 256;
  if (grid > cap) grid = cap;
  rconvert_kernel<RIN, ROUT><<<(unsigned)(grid < 1 ? 1 : grid), 256, 0, current_stream()>>>(p);
  check_launch(kid);
}

}  // namespace qlab
