// qla_ewise.cuh -- the element-wise level-1 families: every output complex
// number depends on the same-position complex number of one or two source
// records (or of the source's adjoint / transpose) and on an optional scalar
// (a constant passed by pointer, or a per-site complex / real field):
//
//   r (eqop) a                      copy, conj, i*a, adjoint, transpose
//   r (eqop) s * b                  s complex or real constant / field, and
//                                   the conj(s), conj(b) forms
//   r = a + b, a - b, s*b + c, s*b - c
//   C / R (eqop) per-site dot products and norms (field outputs)
//   M (eqop) a b^+                  outer product of two ColorVectors
// (lib/perl/build_qla.pl:1256-1335 constant and field multiples, :403-469
// adjoint/transpose/conj copies, :1338-1420 sums and combinations,
// :2358-2460 site-local dot products; QLA complex macro forms
// include/qla_complex.h:140-460).
//
// Map ops run one thread per output complex number: consecutive threads move
// consecutive 8-B (F3) / 16-B (D3) elements of the AoS records, coalesced for
// every record type including the 1152-B DiracPropagator, which does not fit
// one thread's registers.  Each element is computed with the reference's
// macro for its (eqop, form), every multiply and add rounded separately, so
// results are bit-identical.  Local dot products run one thread per site and
// accumulate in FP64 like the reference's QLA_D temporaries.
#pragma once
#include "qla_api.cuh"
#include "qla_launch.cuh"
#include "qla_ops.cuh"

namespace qlab {

enum EwShape : int {
  EW_COPY = 0, EW_CONJ, EW_I, EW_CT, EW_CTA, EW_CAT, EW_CATA, EW_RT, EW_RTA,
  EW_PLUS, EW_MINUS, EW_RT_PLUS, EW_RT_MINUS, EW_CT_PLUS, EW_CT_MINUS
};
enum EwPerm : int { PERM_ID = 0, PERM_M = 1, PERM_P = 2 };     // source element order
enum EwScal : int { SC_NONE = 0, SC_CONST = 1, SC_FIELD = 2 };  // where the scalar comes from

struct EwParams {
  void* out;
  Opnd b, c;           // first and second field source
  Opnd s;              // per-site scalar field (one complex or one real per site)
  const int* gang;
  long long n;
  int eqop;
  const void* sptr;    // constant scalar: device pointer, or nullptr to use sre/sim
  double sre, sim;
};

// element e of a record of the source in the requested order: PERM_M reads
// the transposed 3x3 matrix, PERM_P the spin-colour transposed propagator
template <int PERM, int NE>
__device__ __forceinline__ int perm_elem(int e) {
  if constexpr (PERM == PERM_M) {
    return (e % 3) * 3 + e / 3;
  } else if constexpr (PERM == PERM_P) {
    return (e % 12) * 12 + e / 12;  // (ic,is | jc,js) -> (jc,js | ic,is)
  } else {
    return e;
  }
}

template <typename R>
__device__ __forceinline__ const Cx<R>* rec_ptr(const Opnd& o, long long k, int ne) {
  return (o.mode == OM_PTR) ? static_cast<const Cx<R>*>(o.ptrs[k]) : static_cast<const Cx<R>*>(o.base) + k * ne;
}

template <typename R, int SHAPE>
__device__ __forceinline__ Cx<R> ew_apply(int eqop, Cx<R> x, Cx<R> s, Cx<R> b, Cx<R> c) {
  // t = the value the eq form assigns; peq / meq add / subtract it with one
  // rounding per component; eqm forms are written out as the macros write them
  if constexpr (SHAPE == EW_COPY) {
    switch (eqop) {
      case EQ: return b;
      case EQM: return Cx<R>{-b.re, -b.im};
      case PEQ: return Cx<R>{radd(x.re, b.re), radd(x.im, b.im)};
      default: return Cx<R>{rsub(x.re, b.re), rsub(x.im, b.im)};
    }
  } else if constexpr (SHAPE == EW_CONJ) {
    switch (eqop) {
      case EQ: return Cx<R>{b.re, -b.im};
      case EQM: return Cx<R>{-b.re, b.im};
      case PEQ: return Cx<R>{radd(x.re, b.re), rsub(x.im, b.im)};
      default: return Cx<R>{rsub(x.re, b.re), radd(x.im, b.im)};
    }
  } else if constexpr (SHAPE == EW_I) {
    switch (eqop) {
      case EQ: return Cx<R>{-b.im, b.re};
      case EQM: return Cx<R>{b.im, -b.re};
      case PEQ: return Cx<R>{rsub(x.re, b.im), radd(x.im, b.re)};
      default: return Cx<R>{radd(x.re, b.im), rsub(x.im, b.re)};
    }
  } else if constexpr (SHAPE == EW_RT || SHAPE == EW_RTA) {
    const R tr = rmul(s.re, b.re), ti = rmul(s.re, b.im);
    const R ti_c = SHAPE == EW_RTA ? -ti : ti;  // conj(b): the imaginary part enters negated
    switch (eqop) {
      case EQ: return Cx<R>{tr, ti_c};
      case EQM: return Cx<R>{-tr, -ti_c};
      case PEQ: return SHAPE == EW_RTA ? Cx<R>{radd(x.re, tr), rsub(x.im, ti)} : Cx<R>{radd(x.re, tr), radd(x.im, ti)};
      default: return SHAPE == EW_RTA ? Cx<R>{rsub(x.re, tr), radd(x.im, ti)} : Cx<R>{rsub(x.re, tr), rsub(x.im, ti)};
    }
  } else if constexpr (SHAPE == EW_CT || SHAPE == EW_CTA || SHAPE == EW_CAT || SHAPE == EW_CATA) {
    R re, im;  // the eq-form value
    if constexpr (SHAPE == EW_CT) {
      if (eqop == EQM)
        return Cx<R>{radd(rmul(-s.re, b.re), rmul(s.im, b.im)), rsub(rmul(-s.re, b.im), rmul(s.im, b.re))};
      re = rsub(rmul(s.re, b.re), rmul(s.im, b.im));
      im = radd(rmul(s.re, b.im), rmul(s.im, b.re));
    } else if constexpr (SHAPE == EW_CTA) {  // s * conj(b)
      if (eqop == EQM)
        return Cx<R>{rsub(rmul(-s.re, b.re), rmul(s.im, b.im)), radd(rmul(-s.im, b.re), rmul(s.re, b.im))};
      re = radd(rmul(s.re, b.re), rmul(s.im, b.im));
      im = rsub(rmul(s.im, b.re), rmul(s.re, b.im));
    } else if constexpr (SHAPE == EW_CAT) {  // conj(s) * b
      if (eqop == EQM)
        return Cx<R>{rsub(rmul(-s.re, b.re), rmul(s.im, b.im)), radd(rmul(-s.re, b.im), rmul(s.im, b.re))};
      re = radd(rmul(s.re, b.re), rmul(s.im, b.im));
      im = rsub(rmul(s.re, b.im), rmul(s.im, b.re));
    } else {  // conj(s) * conj(b)
      if (eqop == EQM)
        return Cx<R>{radd(rmul(-s.re, b.re), rmul(s.im, b.im)), radd(rmul(s.re, b.im), rmul(s.im, b.re))};
      re = rsub(rmul(s.re, b.re), rmul(s.im, b.im));
      im = rsub(rmul(-s.re, b.im), rmul(s.im, b.re));
    }
    switch (eqop) {
      case EQ: return Cx<R>{re, im};
      case PEQ: return Cx<R>{radd(x.re, re), radd(x.im, im)};
      default: return Cx<R>{rsub(x.re, re), rsub(x.im, im)};
    }
  } else if constexpr (SHAPE == EW_PLUS) {
    return Cx<R>{radd(b.re, c.re), radd(b.im, c.im)};
  } else if constexpr (SHAPE == EW_MINUS) {
    return Cx<R>{rsub(b.re, c.re), rsub(b.im, c.im)};
  } else if constexpr (SHAPE == EW_RT_PLUS) {
    return Cx<R>{radd(rmul(s.re, b.re), c.re), radd(rmul(s.re, b.im), c.im)};
  } else if constexpr (SHAPE == EW_RT_MINUS) {
    return Cx<R>{rsub(rmul(s.re, b.re), c.re), rsub(rmul(s.re, b.im), c.im)};
  } else if constexpr (SHAPE == EW_CT_PLUS) {
    return Cx<R>{radd(rsub(rmul(s.re, b.re), rmul(s.im, b.im)), c.re),
                 radd(radd(rmul(s.re, b.im), rmul(s.im, b.re)), c.im)};
  } else {  // EW_CT_MINUS
    return Cx<R>{rsub(rsub(rmul(s.re, b.re), rmul(s.im, b.im)), c.re),
                 rsub(radd(rmul(s.re, b.im), rmul(s.im, b.re)), c.im)};
  }
}

template <typename R, int NE, int SHAPE, int PERM, int SCAL, bool SREAL>
__global__ void __launch_bounds__(256) ew_kernel(const EwParams p) {
  constexpr bool TWO = SHAPE == EW_PLUS || SHAPE == EW_MINUS || SHAPE >= EW_RT_PLUS;
  const long long total = p.n * NE;
  const bool load = (p.eqop == PEQ || p.eqop == MEQ);
  Cx<R> sc{R(0), R(0)};
  if constexpr (SCAL == SC_CONST) {
    if (p.sptr) {
      if constexpr (SREAL)
        sc.re = *static_cast<const R*>(p.sptr);
      else
        sc = *static_cast<const Cx<R>*>(p.sptr);
    } else {
      sc = Cx<R>{(R)p.sre, (R)p.sim};
    }
  }
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const long long i = g / NE;
    const int e = (int)(g - i * NE);
    const long long k = p.gang ? (long long)p.gang[i] : i;
    Cx<R> s = sc;
    if constexpr (SCAL == SC_FIELD) {
      if constexpr (SREAL) {
        const R* q = (p.s.mode == OM_PTR) ? static_cast<const R*>(p.s.ptrs[k]) : static_cast<const R*>(p.s.base) + k;
        s.re = *q;
      } else {
        s = *rec_ptr<R>(p.s, k, 1);
      }
    }
    const Cx<R> b = rec_ptr<R>(p.b, k, NE)[perm_elem<PERM, NE>(e)];
    Cx<R> c{R(0), R(0)};
    if constexpr (TWO) c = rec_ptr<R>(p.c, k, NE)[e];
    Cx<R>* out = static_cast<Cx<R>*>(p.out) + k * NE + e;
    const Cx<R> x = load ? *out : Cx<R>{R(0), R(0)};
    *out = ew_apply<R, SHAPE>(p.eqop, x, s, b, c);
  }
}

// Streaming form of the same map when every operand is contiguous and 16-B
// aligned, there is no gang index and no permutation: the records are one
// flat array of n*NE complex numbers, and each thread moves 16-B vectors (two
// F3 / one D3 complex number per vector, two vectors per thread).  A per-site
// scalar field (contiguous) is read for each element's site, element / NE
// (from L1: a site's elements are neighbours).  Element arithmetic is
// ew_apply, so results are identical.
template <typename R, int NE, int SHAPE, int SCAL, bool SREAL>
__global__ void __launch_bounds__(256) ew_flat_kernel(const EwParams p, long long nelem) {
  constexpr bool TWO = SHAPE == EW_PLUS || SHAPE == EW_MINUS || SHAPE >= EW_RT_PLUS;
  constexpr int CPV = 16 / (int)sizeof(Cx<R>);  // complex numbers per 16-B vector
  constexpr int CPT = 2 * CPV;                   // per thread and step
  const bool load = (p.eqop == PEQ || p.eqop == MEQ);
  Cx<R> s{R(0), R(0)};
  if constexpr (SCAL == SC_CONST) {
    if (p.sptr) {
      if constexpr (SREAL)
        s.re = *static_cast<const R*>(p.sptr);
      else
        s = *static_cast<const Cx<R>*>(p.sptr);
    } else {
      s = Cx<R>{(R)p.sre, (R)p.sim};
    }
  }
  const Cx<R>* B = static_cast<const Cx<R>*>(p.b.base);
  const Cx<R>* C = static_cast<const Cx<R>*>(p.c.base);
  Cx<R>* O = static_cast<Cx<R>*>(p.out);
  // the scalar of element q: the constant, or the field at site q / NE
  auto scal_at = [&](long long q) -> Cx<R> {
    if constexpr (SCAL == SC_FIELD) {
      const long long site = q / NE;
      if constexpr (SREAL)
        return Cx<R>{static_cast<const R*>(p.s.base)[site], R(0)};
      else
        return static_cast<const Cx<R>*>(p.s.base)[site];
    } else {
      return s;
    }
  };
  const long long nvec = nelem / CPT;
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nvec;
       v += (long long)gridDim.x * blockDim.x) {
    const long long g0 = v * CPT;
    Cx<R> b[CPT], c[CPT], x[CPT];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const long long q = g0 + h * CPV;
      if constexpr (sizeof(R) == 4) {
        const float4 u = __ldg(reinterpret_cast<const float4*>(B + q));
        b[2 * h] = Cx<R>{u.x, u.y};
        b[2 * h + 1] = Cx<R>{u.z, u.w};
        if constexpr (TWO) {
          const float4 w = __ldg(reinterpret_cast<const float4*>(C + q));
          c[2 * h] = Cx<R>{w.x, w.y};
          c[2 * h + 1] = Cx<R>{w.z, w.w};
        }
        if (load) {
          const float4 o = *reinterpret_cast<const float4*>(O + q);
          x[2 * h] = Cx<R>{o.x, o.y};
          x[2 * h + 1] = Cx<R>{o.z, o.w};
        }
      } else {
        const double2 u = __ldg(reinterpret_cast<const double2*>(B + q));
        b[h] = Cx<R>{u.x, u.y};
        if constexpr (TWO) {
          const double2 w = __ldg(reinterpret_cast<const double2*>(C + q));
          c[h] = Cx<R>{w.x, w.y};
        }
        if (load) {
          const double2 o = *reinterpret_cast<const double2*>(O + q);
          x[h] = Cx<R>{o.x, o.y};
        }
      }
    }
    Cx<R> y[CPT];
#pragma unroll
    for (int j = 0; j < CPT; j++)
      y[j] = ew_apply<R, SHAPE>(p.eqop, load ? x[j] : Cx<R>{R(0), R(0)}, scal_at(g0 + j), b[j], c[j]);
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const long long q = g0 + h * CPV;
      if constexpr (sizeof(R) == 4)
        *reinterpret_cast<float4*>(O + q) = make_float4(y[2 * h].re, y[2 * h].im, y[2 * h + 1].re, y[2 * h + 1].im);
      else
        *reinterpret_cast<double2*>(O + q) = make_double2(y[h].re, y[h].im);
    }
  }
  // tail: the last nelem % CPT numbers, one per thread of the first block
  const long long t0 = nvec * CPT;
  if (blockIdx.x == 0 && t0 + threadIdx.x < nelem) {
    const long long q = t0 + threadIdx.x;
    const Cx<R> x = load ? O[q] : Cx<R>{R(0), R(0)};
    Cx<R> c{R(0), R(0)};
    if constexpr (TWO) c = C[q];
    O[q] = ew_apply<R, SHAPE>(p.eqop, x, scal_at(q), B[q], c);
  }
}

// host side: SCAL_ARG is a pointer to the constant (host or device memory)
// for SC_CONST, ignored otherwise
template <typename R, int NE, int SHAPE, int PERM, int SCAL, bool SREAL>
inline void api_ew(const char* kid, void* r, const void* scal, Opnd s, Opnd b, Opnd c, const int* gang, int n,
                   int eqop) {
  constexpr bool TWO = SHAPE == EW_PLUS || SHAPE == EW_MINUS || SHAPE >= EW_RT_PLUS;
  if (n <= 0) return;
  if (!r || !opnd_ok(b) || (TWO && !opnd_ok(c)) || (SCAL == SC_CONST && !scal) || (SCAL == SC_FIELD && !opnd_ok(s))) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  EwParams p;
  std::memset(&p, 0, sizeof(p));
  p.out = r;
  p.b = b;
  p.c = c;
  p.s = s;
  p.gang = gang;
  p.n = n;
  p.eqop = eqop;
  if constexpr (SCAL == SC_CONST) {
    if (is_device_ptr(scal)) {
      p.sptr = scal;
    } else if constexpr (SREAL) {
      p.sre = (double)*static_cast<const R*>(scal);
    } else {
      p.sre = (double)static_cast<const Cx<R>*>(scal)->re;
      p.sim = (double)static_cast<const Cx<R>*>(scal)->im;
    }
  }
  const long long total = (long long)n * NE;
  const long long cap = (long long)device_sm_count() * 16;
  const bool flat = PERM == PERM_ID && (SCAL != SC_FIELD || s.mode == OM_CONTIG) && gang == nullptr &&
                    b.mode == OM_CONTIG &&
                    (reinterpret_cast<uintptr_t>(b.base) & 15u) == 0 && (reinterpret_cast<uintptr_t>(r) & 15u) == 0 &&
                    (!TWO || (c.mode == OM_CONTIG && (reinterpret_cast<uintptr_t>(c.base) & 15u) == 0));
  if (flat) {
    constexpr int CPT = 2 * (16 / (int)sizeof(Cx<R>));
    long long grid = (total / CPT + 255) / 256;
    if (grid > cap) grid = cap;
    ew_flat_kernel<R, NE, SHAPE, SCAL, SREAL><<<(unsigned)(grid < 1 ? 1 : grid), 256, 0, current_stream()>>>(p, total);
  } else {
    long long grid = (total + 255) / 256;
    if (grid > cap) grid = cap;
    ew_kernel<R, NE, SHAPE, PERM, SCAL, SREAL><<<(unsigned)(grid < 1 ? 1 : grid), 256, 0, current_stream()>>>(p);
  }
  check_launch(kid);
}

// ---------------------------------------------------------------------------
// outer product M (eqop) a b^+ of two ColorVectors (one thread per element)
template <typename R>
__global__ void __launch_bounds__(256) outer_kernel(const EwParams p) {
  const long long total = p.n * 9;
  const bool load = (p.eqop == PEQ || p.eqop == MEQ);
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const long long i = g / 9;
    const int e = (int)(g - i * 9);
    const long long k = p.gang ? (long long)p.gang[i] : i;
    const Cx<R> a = rec_ptr<R>(p.b, k, 3)[e / 3];
    const Cx<R> b = rec_ptr<R>(p.c, k, 3)[e % 3];
    Cx<R>* out = static_cast<Cx<R>*>(p.out) + k * 9 + e;
    const Cx<R> x = load ? *out : Cx<R>{R(0), R(0)};
    // c_(eqop)_c_times_ca(r, a, b): the scalar slot carries a
    *out = ew_apply<R, EW_CTA>(p.eqop, x, a, b, Cx<R>{R(0), R(0)});
  }
}

template <typename R>
inline void api_outer(const char* kid, void* r, Opnd a, Opnd b, const int* gang, int n, int eqop) {
  if (n <= 0) return;
  if (!r || !opnd_ok(a) || !opnd_ok(b)) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  EwParams p;
  std::memset(&p, 0, sizeof(p));
  p.out = r;
  p.b = a;
  p.c = b;
  p.gang = gang;
  p.n = n;
  p.eqop = eqop;
  long long grid = ((long long)n * 9 + 255) / 256;
  const long long cap = (long long)device_sm_count() * 16;
  if (grid > cap) grid = cap;
  outer_kernel<R><<<(unsigned)(grid < 1 ? 1 : grid), 256, 0, current_stream()>>>(p);
  check_launch(kid);
}

// ---------------------------------------------------------------------------
// site-local dot products and norms (field outputs), one thread per site
enum LdKind : int { LD_DOT = 0, LD_DOT_AA = 1, LD_ADOT = 2, LD_REDOT = 3, LD_NORM2 = 4 };
// LD_DOT    x += conj(a_e) b_e                 (X_dot_X)
// LD_DOT_AA x += conj(a_e) conj(b_perm(e))     (M_dot_Ma, P_dot_Pa)
// LD_ADOT   x += a_perm(e) b_e                 (Ma_dot_M, Pa_dot_P)
// LD_REDOT  x += Re(conj(a_e) b_e)             (re_X_dot_X)
// LD_NORM2  x += |a_e|^2                       (norm2_X)

// The accumulation of one site shared by the two kernels below: x over the
// elements e in order, from the records a and b (any memory space)
template <typename R, int NE, int KIND, int PERM>
__device__ __forceinline__ void ldot_site(const Cx<R>* a, const Cx<R>* b, double& xr, double& xi) {
  xr = 0.0;
  xi = 0.0;
#pragma unroll 4
  for (int e = 0; e < NE; e++) {
    Cx<R> ua = a[e], vb = b[e];
    if constexpr (KIND == LD_ADOT) ua = a[perm_elem<PERM, NE>(e)];
    if constexpr (KIND == LD_DOT_AA) vb = b[perm_elem<PERM, NE>(e)];
    const double ur = ua.re, ui = ua.im, vr = vb.re, vi = vb.im;
    if constexpr (KIND == LD_DOT || KIND == LD_REDOT || KIND == LD_NORM2) {
      xr = __dadd_rn(xr, __dadd_rn(__dmul_rn(ur, vr), __dmul_rn(ui, vi)));
      if constexpr (KIND == LD_DOT) xi = __dadd_rn(xi, __dsub_rn(__dmul_rn(ur, vi), __dmul_rn(ui, vr)));
    } else if constexpr (KIND == LD_DOT_AA) {
      xr = __dadd_rn(xr, __dsub_rn(__dmul_rn(ur, vr), __dmul_rn(ui, vi)));
      xi = __dadd_rn(xi, __dsub_rn(__dmul_rn(-ur, vi), __dmul_rn(ui, vr)));
    } else {
      xr = __dadd_rn(xr, __dsub_rn(__dmul_rn(ur, vr), __dmul_rn(ui, vi)));
      xi = __dadd_rn(xi, __dadd_rn(__dmul_rn(ur, vi), __dmul_rn(ui, vr)));
    }
  }
}

template <typename R, int KIND>
__device__ __forceinline__ void ldot_store(void* out, long long k, int eqop, double xr, double xi) {
  if constexpr (KIND >= LD_REDOT) {
    R* q = static_cast<R*>(out) + k;
    switch (eqop) {
      case EQ: *q = (R)xr; break;
      case EQM: *q = (R)(-xr); break;
      case PEQ: *q = (R)__dadd_rn((double)*q, xr); break;
      default: *q = (R)__dsub_rn((double)*q, xr); break;
    }
  } else {
    Cx<R>* q = static_cast<Cx<R>*>(out) + k;
    const Cx<R> t{(R)xr, (R)xi};
    switch (eqop) {
      case EQ: *q = t; break;
      case EQM: *q = Cx<R>{-t.re, -t.im}; break;
      case PEQ: *q = Cx<R>{radd(q->re, t.re), radd(q->im, t.im)}; break;
      default: *q = Cx<R>{rsub(q->re, t.re), rsub(q->im, t.im)}; break;
    }
  }
}

// Staged form for contiguous operands without a gang index: a block copies
// the records of S consecutive sites with coalesced loads (LD_U in flight
// per thread) into shared memory (rows padded by one complex number against
// bank conflicts), then each of the first S threads accumulates its site
// from there.  (Per-thread cp.async copies in two stages measured slower
// than this on B200: 0.75 against 0.88 of HBM for the D3 D dot product.)
// one thread per site, records read where they are (gang or pointer forms)
template <typename R, int NE, int KIND, int PERM>
__global__ void __launch_bounds__(256) ldot_kernel(const EwParams p) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < p.n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long k = p.gang ? (long long)p.gang[i] : i;
    const Cx<R>* a = rec_ptr<R>(p.b, k, NE);
    const Cx<R>* b = (KIND == LD_NORM2) ? a : rec_ptr<R>(p.c, k, NE);
    double xr, xi;
    ldot_site<R, NE, KIND, PERM>(a, b, xr, xi);
    ldot_store<R, KIND>(p.out, k, p.eqop, xr, xi);
  }
}

template <typename R, int NE, int KIND, int PERM, int S>
__global__ void __launch_bounds__(128) ldot_smem_kernel(const EwParams p) {
  extern __shared__ __align__(16) unsigned char ldsm[];
  constexpr int ST = NE + 1;  // padded row stride (complex numbers)
  Cx<R>* sa = reinterpret_cast<Cx<R>*>(ldsm);
  Cx<R>* sb = sa + S * ST;
  const Cx<R>* A = static_cast<const Cx<R>*>(p.b.base);
  const Cx<R>* B = static_cast<const Cx<R>*>(KIND == LD_NORM2 ? p.b.base : p.c.base);
  const long long ntile = (p.n + S - 1) / S;
  for (long long tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const long long s0 = tile * S;
    const int ns = (int)((p.n - s0) < S ? (p.n - s0) : S);
    const long long base = s0 * NE;
    const int nf = ns * NE;
    // LD_U loads per thread issued before their shared-memory stores, so
    // that many are in flight (a load-store loop would wait for each)
    constexpr int LD_U = 12;
    for (int f0 = threadIdx.x; f0 < nf; f0 += LD_U * blockDim.x) {
      Cx<R> va[LD_U], vb[LD_U];
#pragma unroll
      for (int u = 0; u < LD_U; u++) {
        const int f = f0 + u * blockDim.x;
        if (f < nf) {
          va[u] = A[base + f];
          if constexpr (KIND != LD_NORM2) vb[u] = B[base + f];
        }
      }
#pragma unroll
      for (int u = 0; u < LD_U; u++) {
        const int f = f0 + u * blockDim.x;
        if (f < nf) {
          const int row = f / NE, col = f - row * NE;
          sa[row * ST + col] = va[u];
          if constexpr (KIND != LD_NORM2) sb[row * ST + col] = vb[u];
        }
      }
    }
    __syncthreads();
    if (threadIdx.x < ns) {
      double xr, xi;
      const Cx<R>* ra = sa + threadIdx.x * ST;
      ldot_site<R, NE, KIND, PERM>(ra, KIND == LD_NORM2 ? ra : sb + threadIdx.x * ST, xr, xi);
      ldot_store<R, KIND>(p.out, s0 + threadIdx.x, p.eqop, xr, xi);
    }
    __syncthreads();
  }
}

template <typename R, int NE, int KIND, int PERM>
inline void api_ldot(const char* kid, void* r, Opnd a, Opnd b, const int* gang, int n, int eqop) {
  if (n <= 0) return;
  if (!r || !opnd_ok(a) || (KIND != LD_NORM2 && !opnd_ok(b))) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  EwParams p;
  std::memset(&p, 0, sizeof(p));
  p.out = r;
  p.b = a;
  p.c = b;
  p.gang = gang;
  p.n = n;
  p.eqop = eqop;
  const long long cap = (long long)device_sm_count() * 16;
  if (gang == nullptr && a.mode == OM_CONTIG && (KIND == LD_NORM2 || b.mode == OM_CONTIG)) {
    constexpr int S = NE > 32 ? 32 : 128;
    const size_t smem = (size_t)(KIND == LD_NORM2 ? 1 : 2) * S * (NE + 1) * sizeof(Cx<R>);
    const void* fn = reinterpret_cast<const void*>(&ldot_smem_kernel<R, NE, KIND, PERM, S>);
    static bool attr_set[64] = {false};
    const int dev = current_device();
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      attr_set[dev] = true;
    }
    long long grid = ((long long)n + S - 1) / S;
    if (grid > cap) grid = cap;
    ldot_smem_kernel<R, NE, KIND, PERM, S><<<(unsigned)(grid < 1 ? 1 : grid), 128, smem, current_stream()>>>(p);
  } else {
    long long grid = ((long long)n + 255) / 256;
    if (grid > cap) grid = cap;
    ldot_kernel<R, NE, KIND, PERM><<<(unsigned)(grid < 1 ? 1 : grid), 256, 0, current_stream()>>>(p);
  }
  check_launch(kid);
}

}  // namespace qlab
