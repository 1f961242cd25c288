// qla_ncolor.cuh -- the element-wise, site-local product, fill / component /
// gamma / trace families and the global P / adjoint-form reductions, sums
// and precision conversions of QLA_FN_ / QLA_DN_ / QLA_DFN_ (colour count nc
// chosen at run time, doc/qla.tex:595-611).
//
// These are the families of qla_ewise.cuh and qla_sitefield.cuh with the
// record length and the colour count as kernel arguments instead of
// template parameters, so one kernel serves every nc the caller passes (the
// reference's N-colour libraries take any nc).  The arithmetic of every
// element is the same device function as in the fixed-colour kernels
// (ew_apply, ldot accumulation order, phase_times), so results are
// bit-identical to the reference's N-colour code.
//
// Index arithmetic: a grid-stride loop over the n * ne output elements
// divides its starting index once and then steps (site, element) by the
// constant stride; colour / spin positions inside a record are split with
// div_small (a float-reciprocal quotient with one integer correction, exact
// for the record sizes here).
#pragma once
#include <vector>
#include "qla_sitefield.cuh"
#include "qla_prop.cuh"
#include "qla_multi.cuh"

namespace qlab {

// floor(e / d) for 0 <= e < 2^22, 1 <= d <= 2^10: the float product is
// within 2^-1 of e / d, so one correction step makes it exact
__device__ __forceinline__ int div_small(int e, int d, float inv) {
  int q = __float2int_rz(__int2float_rn(e) * inv);
  const int r = e - q * d;
  if (r < 0)
    q--;
  else if (r >= d)
    q++;
  return q;
}

// element of the source read for output element e: PERM_M transposes the
// nc x nc matrix, PERM_P the (4 nc) x (4 nc) propagator
__device__ __forceinline__ int perm_elem_n(int perm, int e, int blk, float inv_blk) {
  if (perm == PERM_ID) return e;
  const int q = div_small(e, blk, inv_blk);
  return (e - q * blk) * blk + q;
}

struct NcDims {
  int nc;        // colours
  int ne;        // complex numbers per record of the field being mapped
  int perm;      // EwPerm of the source
  int blk;       // row length of the permuted record (nc for M, 4 nc for P)
  float inv_blk;
};

inline NcDims nc_dims(int nc, int ne, int perm) {
  NcDims d;
  d.nc = nc;
  d.ne = ne;
  d.perm = perm;
  d.blk = (perm == PERM_P) ? 4 * nc : nc;
  d.inv_blk = 1.0f / (float)d.blk;
  return d;
}

// grid-stride walk over (site i, element e) pairs without a division per step
struct SiteElemWalk {
  long long i;
  int e;
  long long si;
  int se;
  __device__ __forceinline__ SiteElemWalk(int ne) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long S = (long long)gridDim.x * blockDim.x;
    i = g / ne;
    e = (int)(g - i * ne);
    si = S / ne;
    se = (int)(S - si * ne);
  }
  __device__ __forceinline__ void next(int ne) {
    i += si;
    e += se;
    if (e >= ne) {
      e -= ne;
      i++;
    }
  }
};

inline unsigned nc_grid(long long total) {
  const long long cap = (long long)device_sm_count() * 16;
  long long grid = (total + 255) / 256;
  if (grid > cap) grid = cap;
  return (unsigned)(grid < 1 ? 1 : grid);
}

inline bool nc_ok(const char* kid, int nc) {
  if (nc < 1 || nc > 64) {
    set_error(QLAGPU_ERR_ARG, kid, "nc outside 1..64");
    return false;
  }
  return true;
}

// ---------------------------------------------------------------------------
// element-wise families (qla_ewise.cuh api_ew with run-time ne / perm)
template <typename R, int SHAPE, int SCAL, bool SREAL>
__global__ void __launch_bounds__(256) ewn_kernel(const EwParams p, const NcDims d) {
  constexpr bool TWO = SHAPE == EW_PLUS || SHAPE == EW_MINUS || SHAPE >= EW_RT_PLUS;
  const bool load = (p.eqop == PEQ || p.eqop == MEQ);
  const int ne = d.ne;
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
  for (SiteElemWalk w(ne); w.i < p.n; w.next(ne)) {
    const long long k = p.gang ? (long long)p.gang[w.i] : w.i;
    Cx<R> s = sc;
    if constexpr (SCAL == SC_FIELD) {
      if constexpr (SREAL) {
        const R* q = (p.s.mode == OM_PTR) ? static_cast<const R*>(p.s.ptrs[k]) : static_cast<const R*>(p.s.base) + k;
        s.re = *q;
      } else {
        s = *rec_ptr<R>(p.s, k, 1);
      }
    }
    const Cx<R> b = rec_ptr<R>(p.b, k, ne)[perm_elem_n(d.perm, w.e, d.blk, d.inv_blk)];
    Cx<R> c{R(0), R(0)};
    if constexpr (TWO) c = rec_ptr<R>(p.c, k, ne)[w.e];
    Cx<R>* out = static_cast<Cx<R>*>(p.out) + k * ne + w.e;
    const Cx<R> x = load ? *out : Cx<R>{R(0), R(0)};
    *out = ew_apply<R, SHAPE>(p.eqop, x, s, b, c);
  }
}

template <typename R, int SHAPE, int SCAL, bool SREAL>
inline void api_ew_n(const char* kid, int nc, int ne, int perm, void* r, const void* scal, Opnd s, Opnd b, Opnd c,
                     const int* gang, int n, int eqop) {
  constexpr bool TWO = SHAPE == EW_PLUS || SHAPE == EW_MINUS || SHAPE >= EW_RT_PLUS;
  if (!nc_ok(kid, nc) || n <= 0) return;
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
  ewn_kernel<R, SHAPE, SCAL, SREAL><<<nc_grid((long long)n * ne), 256, 0, current_stream()>>>(p, nc_dims(nc, ne, perm));
  check_launch(kid);
}

// outer product M (eqop) a b^+ of two nc-vectors
template <typename R>
__global__ void __launch_bounds__(256) outern_kernel(const EwParams p, int nc) {
  const int m = nc * nc;
  const float inv = 1.0f / (float)nc;
  const bool load = (p.eqop == PEQ || p.eqop == MEQ);
  for (SiteElemWalk w(m); w.i < p.n; w.next(m)) {
    const long long k = p.gang ? (long long)p.gang[w.i] : w.i;
    const int ic = div_small(w.e, nc, inv), jc = w.e - ic * nc;
    const Cx<R> a = rec_ptr<R>(p.b, k, nc)[ic];
    const Cx<R> b = rec_ptr<R>(p.c, k, nc)[jc];
    Cx<R>* out = static_cast<Cx<R>*>(p.out) + k * m + w.e;
    const Cx<R> x = load ? *out : Cx<R>{R(0), R(0)};
    *out = ew_apply<R, EW_CTA>(p.eqop, x, a, b, Cx<R>{R(0), R(0)});
  }
}

template <typename R>
inline void api_outer_n(const char* kid, int nc, void* r, Opnd a, Opnd b, const int* gang, int n, int eqop) {
  if (!nc_ok(kid, nc) || n <= 0) return;
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
  outern_kernel<R><<<nc_grid((long long)n * nc * nc), 256, 0, current_stream()>>>(p, nc);
  check_launch(kid);
}

// ---------------------------------------------------------------------------
// site-local dot products and norms: ldot_site's accumulation with run-time
// record length; the permuted forms walk the transposed source row by row
template <typename R, int KIND>
__device__ __forceinline__ void ldot_site_n(const Cx<R>* a, const Cx<R>* b, const NcDims& d, double& xr,
                                            double& xi) {
  xr = 0.0;
  xi = 0.0;
  const bool perm = (KIND == LD_ADOT || KIND == LD_DOT_AA);
  const int B = perm ? d.blk : 1;
  const int rows = perm ? d.blk : 1, cols = perm ? d.blk : d.ne;
  for (int x = 0; x < rows; x++)
    for (int y = 0; y < cols; y++) {
      const int e = x * cols + y;
      const int pe = perm ? y * B + x : e;
      Cx<R> ua = a[e], vb = b[e];
      if constexpr (KIND == LD_ADOT) ua = a[pe];
      if constexpr (KIND == LD_DOT_AA) vb = b[pe];
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
__global__ void __launch_bounds__(256) ldotn_kernel(const EwParams p, const NcDims d) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < p.n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long k = p.gang ? (long long)p.gang[i] : i;
    const Cx<R>* a = rec_ptr<R>(p.b, k, d.ne);
    const Cx<R>* b = (KIND == LD_NORM2) ? a : rec_ptr<R>(p.c, k, d.ne);
    double xr, xi;
    ldot_site_n<R, KIND>(a, b, d, xr, xi);
    ldot_store<R, KIND>(p.out, k, p.eqop, xr, xi);
  }
}

template <typename R, int KIND>
inline void api_ldot_n(const char* kid, int nc, int ne, int perm, void* r, Opnd a, Opnd b, const int* gang, int n,
                       int eqop) {
  if (!nc_ok(kid, nc) || n <= 0) return;
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
  ldotn_kernel<R, KIND><<<nc_grid(n), 256, 0, current_stream()>>>(p, nc_dims(nc, ne, perm));
  check_launch(kid);
}

// ---------------------------------------------------------------------------
// fills, copymask, components, gamma, trace, antihermitian part

struct SfnParams {
  void* out;
  Opnd a, m;
  const int* gang;
  long long n;
  int eqop, nc, ne_out, ne_src;
  int what;              // SF_SUB: 'e', 'c', 'd'
  char dst, src, cont;   // SF_SUB: record letters
  int i_c, i_s, j_c, j_s;
  int gs[4], gp[4];
  const void* cptr;      // constant record / number in device memory
};

// component of (ic, is, jc, js) in a record of letter t with nc colours
__host__ __device__ __forceinline__ int elem_n(char t, int nc, int ic, int is, int jc, int js) {
  switch (t) {
    case 'V': return ic;
    case 'H': return ic * 2 + is;
    case 'D': return ic * 4 + is;
    case 'M': return ic * nc + jc;
    case 'P': return ((ic * 4 + is) * nc + jc) * 4 + js;
    default: return 0;
  }
}

inline int ne_of_letter(char t, int nc) {
  switch (t) {
    case 'V': return nc;
    case 'H': return 2 * nc;
    case 'D': return 4 * nc;
    case 'M': return nc * nc;
    case 'P': return 16 * nc * nc;
    default: return 1;
  }
}

// output elements per site of each kind
__device__ __forceinline__ int sfn_ops(const SfnParams& p, int KIND) {
  if (KIND == SF_TRACE_C || KIND == SF_TRACE_RE || KIND == SF_TRACE_IM) return 1;
  if (KIND == SF_SUB) return p.what == 'e' ? 1 : (p.what == 'c' ? p.nc : 4 * p.nc);
  return p.ne_out;
}

template <typename R, int KIND>
__global__ void __launch_bounds__(256) sfn_kernel(const SfnParams p) {
  const int ops = sfn_ops(p, KIND);
  const int nc = p.nc;
  const float inv_nc = 1.0f / (float)nc, inv_4nc = 1.0f / (float)(4 * nc);
  Cx<R> c1{R(0), R(0)};
  if constexpr (KIND == SF_DIAG) c1 = *static_cast<const Cx<R>*>(p.cptr);
  for (SiteElemWalk w(ops); w.i < p.n; w.next(ops)) {
    const long long k = p.gang ? (long long)p.gang[w.i] : w.i;
    const int e = w.e;
    if constexpr (KIND == SF_BCAST) {
      Cx<R>* out = static_cast<Cx<R>*>(p.out) + k * p.ne_out + e;
      const Cx<R> b = static_cast<const Cx<R>*>(p.cptr)[e];
      const bool load = (p.eqop == PEQ || p.eqop == MEQ);
      const Cx<R> x = load ? *out : Cx<R>{R(0), R(0)};
      *out = ew_apply<R, EW_COPY>(p.eqop, x, Cx<R>{R(0), R(0)}, b, Cx<R>{R(0), R(0)});
    } else if constexpr (KIND == SF_DIAG) {
      Cx<R>* out = static_cast<Cx<R>*>(p.out) + k * p.ne_out + e;
      Cx<R> x;
      switch (p.eqop) {
        case EQ: x = Cx<R>{R(0), R(0)}; break;
        case EQM: x = Cx<R>{-R(0), R(0)}; break;
        case PEQ: x = *out; x.re = radd(x.re, R(0)); break;
        default: x = *out; x.re = rsub(x.re, R(0)); break;
      }
      const int ic = div_small(e, nc, inv_nc);
      if (e - ic * nc == ic) {
        switch (p.eqop) {
          case EQ: x = c1; break;
          case EQM: x = Cx<R>{-c1.re, -c1.im}; break;
          case PEQ: x = Cx<R>{radd(x.re, c1.re), radd(x.im, c1.im)}; break;
          default: x = Cx<R>{rsub(x.re, c1.re), rsub(x.im, c1.im)}; break;
        }
      }
      *out = x;
    } else if constexpr (KIND == SF_ZERO) {
      static_cast<Cx<R>*>(p.out)[k * p.ne_out + e] = Cx<R>{R(0), R(0)};
    } else if constexpr (KIND == SF_MASK) {
      const int mv = (p.m.mode == OM_PTR) ? *static_cast<const int*>(p.m.ptrs[k]) : static_cast<const int*>(p.m.base)[k];
      if (mv) static_cast<Cx<R>*>(p.out)[k * p.ne_out + e] = rec_ptr<R>(p.a, k, p.ne_src)[e];
    } else if constexpr (KIND == SF_SUB) {
      int o, s;
      if (p.what == 'e') {
        o = (p.dst == 'C') ? 0 : elem_n(p.dst, nc, p.i_c, p.i_s, p.j_c, p.j_s);
        s = (p.src == 'C') ? 0 : elem_n(p.src, nc, p.i_c, p.i_s, p.j_c, p.j_s);
      } else if (p.what == 'c') {
        const int ce = elem_n(p.cont, nc, e, p.i_s, p.j_c, p.j_s);
        o = (p.dst == 'V') ? e : ce;
        s = (p.src == 'V') ? e : ce;
      } else {
        const int ic = e >> 2, is = e & 3;
        const int pe = elem_n('P', nc, ic, is, p.j_c, p.j_s);
        o = (p.dst == 'D') ? e : pe;
        s = (p.src == 'D') ? e : pe;
      }
      static_cast<Cx<R>*>(p.out)[k * p.ne_out + o] = rec_ptr<R>(p.a, k, p.ne_src)[s];
    } else if constexpr (KIND == SF_GAMMA_L || KIND == SF_GAMMA_R) {
      int s, base, stride;
      if (KIND == SF_GAMMA_R || p.ne_out == 4 * nc) {
        s = e & 3;
        base = e - s;
        stride = 1;
      } else {
        // P: e = (ic*4 + is) * 4nc + (jc*4 + js)
        const int row = div_small(e, 4 * nc, inv_4nc);
        s = row & 3;
        base = e - s * 4 * nc;
        stride = 4 * nc;
      }
      const Cx<R> a = rec_ptr<R>(p.a, k, p.ne_src)[base + p.gs[s] * stride];
      static_cast<Cx<R>*>(p.out)[k * p.ne_out + e] = phase_times<R>(p.gp[s], a);
    } else if constexpr (KIND == SF_TRACE_C) {
      const Cx<R>* a = rec_ptr<R>(p.a, k, nc * nc);
      Cx<R> x{R(0), R(0)};
      for (int c = 0; c < nc; c++) x = Cx<R>{radd(x.re, a[c * (nc + 1)].re), radd(x.im, a[c * (nc + 1)].im)};
      static_cast<Cx<R>*>(p.out)[k] = x;
    } else if constexpr (KIND == SF_TRACE_RE || KIND == SF_TRACE_IM) {
      const Cx<R>* a = rec_ptr<R>(p.a, k, nc * nc);
      R x = R(0);
      for (int c = 0; c < nc; c++) x = radd(x, KIND == SF_TRACE_RE ? a[c * (nc + 1)].re : a[c * (nc + 1)].im);
      static_cast<R*>(p.out)[k] = x;
    } else {  // SF_ANTIHERM
      const Cx<R>* a = rec_ptr<R>(p.a, k, nc * nc);
      const int ic = div_small(e, nc, inv_nc), jc = e - ic * nc;
      Cx<R> y;
      if (ic == jc) {
        R x = R(0);
        for (int c = 0; c < nc; c++) x = radd(x, a[c * (nc + 1)].im);
        x = rdiv(x, (R)nc);
        y = Cx<R>{R(0), rsub(a[e].im, x)};
      } else {
        const int lo = ic < jc ? ic : jc, hi = ic < jc ? jc : ic;
        const Cx<R> u = a[lo * nc + hi], v = a[hi * nc + lo];
        const Cx<R> x2{rmul(rsub(u.re, v.re), R(0.5)), rmul(radd(u.im, v.im), R(0.5))};
        y = (ic < jc) ? x2 : Cx<R>{-x2.re, x2.im};
      }
      static_cast<Cx<R>*>(p.out)[k * nc * nc + e] = y;
    }
  }
}

inline bool sfn_prep(const char* kid, SfnParams& p, int nc, void* r, Opnd a, const int* gang, int n, int eqop,
                     bool need_a) {
  if (!nc_ok(kid, nc) || n <= 0) return false;
  if (!r || (need_a && !opnd_ok(a))) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return false;
  }
  std::memset(&p, 0, sizeof(p));
  p.out = r;
  p.a = a;
  p.gang = gang;
  p.n = n;
  p.eqop = eqop;
  p.nc = nc;
  return true;
}

template <typename R, int KIND>
inline void sfn_launch(const char* kid, const SfnParams& p, long long ops) {
  sfn_kernel<R, KIND><<<nc_grid(p.n * ops), 256, 0, current_stream()>>>(p);
  check_launch(kid);
}

// a constant of `bytes` bytes in host or device memory, made device-resident
// for the launch: a host constant is copied into a stream-ordered allocation
// that is released after the kernel on the same stream
struct DevConst {
  const void* ptr = nullptr;
  void* owned = nullptr;
  bool make(const char* kid, const void* x, size_t bytes) {
    if (is_device_ptr(x)) {
      ptr = x;
      return true;
    }
    cudaStream_t st = current_stream();
    if (cudaMallocAsync(&owned, bytes, st) != cudaSuccess) {
      cudaGetLastError();
      set_error(QLAGPU_ERR_ALLOC, kid, "stream-ordered allocation of the constant failed");
      return false;
    }
    if (cudaMemcpyAsync(owned, x, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) {
      check_launch(kid);
      return false;
    }
    ptr = owned;
    return true;
  }
  ~DevConst() {
    if (owned) cudaFreeAsync(owned, current_stream());
  }
};

template <typename R>
inline void api_fill_n(const char* kid, int nc, int ne, void* r, const void* x, const int* gang, int n, int eqop) {
  SfnParams p;
  if (!sfn_prep(kid, p, nc, r, Opnd{}, gang, n, eqop, false)) return;
  if (!x) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  DevConst c;
  if (!c.make(kid, x, (size_t)ne * sizeof(Cx<R>))) return;
  p.cptr = c.ptr;
  p.ne_out = p.ne_src = ne;
  sfn_launch<R, SF_BCAST>(kid, p, ne);
}

template <typename R>
inline void api_diagfill_n(const char* kid, int nc, void* r, const void* cv, const int* gang, int n, int eqop) {
  SfnParams p;
  if (!sfn_prep(kid, p, nc, r, Opnd{}, gang, n, eqop, false)) return;
  if (!cv) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  DevConst c;
  if (!c.make(kid, cv, sizeof(Cx<R>))) return;
  p.cptr = c.ptr;
  p.ne_out = p.ne_src = nc * nc;
  sfn_launch<R, SF_DIAG>(kid, p, (long long)nc * nc);
}

template <typename R>
inline void api_zero_n(const char* kid, int nc, int ne, void* r, const int* gang, int n) {
  SfnParams p;
  if (!sfn_prep(kid, p, nc, r, Opnd{}, gang, n, EQ, false)) return;
  p.ne_out = p.ne_src = ne;
  sfn_launch<R, SF_ZERO>(kid, p, ne);
}

template <typename R>
inline void api_mask_n(const char* kid, int nc, int ne, void* r, Opnd a, Opnd m, const int* gang, int n) {
  SfnParams p;
  if (!sfn_prep(kid, p, nc, r, a, gang, n, EQ, true)) return;
  if (!opnd_ok(m)) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  p.m = m;
  p.ne_out = p.ne_src = ne;
  sfn_launch<R, SF_MASK>(kid, p, ne);
}

template <typename R>
inline void api_sub_n(const char* kid, int nc, void* r, Opnd a, const int* gang, int n, char what, char dst, char src,
                      int i_c, int i_s, int j_c, int j_s) {
  SfnParams p;
  if (!sfn_prep(kid, p, nc, r, a, gang, n, EQ, true)) return;
  const char cont = (dst == 'V' || dst == 'C' || (what == 'd' && dst == 'D')) ? src : dst;
  if (i_c < 0 || i_c >= nc || i_s < 0 || i_s > (cont == 'H' ? 1 : 3) || j_c < 0 || j_c >= nc || j_s < 0 || j_s > 3) {
    set_error(QLAGPU_ERR_ARG, kid, "colour or spin index out of range");
    return;
  }
  p.what = what;
  p.dst = dst;
  p.src = src;
  p.cont = cont;
  p.i_c = i_c;
  p.i_s = i_s;
  p.j_c = j_c;
  p.j_s = j_s;
  p.ne_out = ne_of_letter(dst, nc);
  p.ne_src = ne_of_letter(src, nc);
  sfn_launch<R, SF_SUB>(kid, p, what == 'e' ? 1 : (what == 'c' ? nc : 4 * nc));
}

template <typename R, bool LEFT>
inline void api_gamma_n(const char* kid, int nc, int ne, void* r, Opnd a, int mu, const int* gang, int n) {
  if (mu < 0 || mu > 15) {
    std::printf("Gamma matrix %d not supported\n", mu);
    set_error(QLAGPU_ERR_ARG, kid, "gamma matrix index outside 0..15");
    return;
  }
  SfnParams p;
  if (!sfn_prep(kid, p, nc, r, a, gang, n, EQ, true)) return;
  const GammaTable& t = gamma_table();
  for (int s = 0; s < 4; s++) {
    p.gs[s] = LEFT ? t.row_src[mu][s] : t.col_src[mu][s];
    p.gp[s] = LEFT ? t.row_ph[mu][s] : t.col_ph[mu][s];
  }
  p.ne_out = p.ne_src = ne;
  if constexpr (LEFT)
    sfn_launch<R, SF_GAMMA_L>(kid, p, ne);
  else
    sfn_launch<R, SF_GAMMA_R>(kid, p, ne);
}

template <typename R, int KIND>
inline void api_trace_n(const char* kid, int nc, void* r, Opnd a, const int* gang, int n) {
  SfnParams p;
  if (!sfn_prep(kid, p, nc, r, a, gang, n, EQ, true)) return;
  p.ne_out = 1;
  p.ne_src = nc * nc;
  sfn_launch<R, KIND>(kid, p, 1);
}

template <typename R>
inline void api_antiherm_n(const char* kid, int nc, void* r, Opnd a, const int* gang, int n) {
  SfnParams p;
  if (!sfn_prep(kid, p, nc, r, a, gang, n, EQ, true)) return;
  p.ne_out = p.ne_src = nc * nc;
  sfn_launch<R, SF_ANTIHERM>(kid, p, (long long)nc * nc);
}

// ---------------------------------------------------------------------------
// global reductions of P and of the adjoint forms, one thread per site
template <typename R, int KIND, typename OUT>
__global__ void __launch_bounds__(256) gdotn_kernel(const EwParams p, const SiteParams rp, const NcDims d) {
  using FIN = GDotFinish<KIND, OUT>;
  DD acc[ArrN<FIN::NACC>::value];
#pragma unroll
  for (int a = 0; a < ArrN<FIN::NACC>::value; a++) acc[a] = DD{0.0, 0.0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < p.n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long k = p.gang ? (long long)p.gang[i] : i;
    const Cx<R>* a = rec_ptr<R>(p.b, k, d.ne);
    const Cx<R>* b = (KIND == LD_NORM2) ? a : rec_ptr<R>(p.c, k, d.ne);
    double xr, xi;
    ldot_site_n<R, KIND>(a, b, d, xr, xi);
    dd_add(acc[0], xr);
    if constexpr (FIN::NACC > 1) dd_add(acc[1], xi);
  }
  reduce_finish<FIN>(rp, acc);
}

// contiguous fields without a gang index: one flat stream of complex
// numbers (gdot_flat_kernel's scheme with a run-time record length; the
// unpermuted forms need no element positions and take its grouped sums)
template <typename R, int KIND, typename OUT>
__global__ void __launch_bounds__(256, 4) gdotn_flat_kernel(const EwParams p, const SiteParams rp, const NcDims d) {
  using FIN = GDotFinish<KIND, OUT>;
  if constexpr (KIND == LD_DOT || KIND == LD_REDOT || KIND == LD_NORM2) {
    DD acc[ArrN<FIN::NACC>::value];
#pragma unroll
    for (int a = 0; a < ArrN<FIN::NACC>::value; a++) acc[a] = DD{0.0, 0.0};
    const Cx<R>* A = static_cast<const Cx<R>*>(p.b.base);
    const Cx<R>* B = static_cast<const Cx<R>*>(KIND == LD_NORM2 ? p.b.base : p.c.base);
    const long long total = p.n * d.ne;
    const long long stride = (long long)gridDim.x * blockDim.x;
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (; g + (GD_U - 1) * stride < total; g += GD_U * stride) {
      double tr[GD_U], ti[GD_U];
#pragma unroll
      for (int u = 0; u < GD_U; u++) gdot_term<R, 1, KIND, 0>(A + g + u * stride, B + g + u * stride, 0, tr[u], ti[u]);
      dd_add(acc[0], tree_sum(tr));
      if constexpr (FIN::NACC > 1) dd_add(acc[1], tree_sum(ti));
    }
    for (; g < total; g += stride) {
      double tr, ti;
      gdot_term<R, 1, KIND, 0>(A + g, B + g, 0, tr, ti);
      dd_add(acc[0], tr);
      if constexpr (FIN::NACC > 1) dd_add(acc[1], ti);
    }
    reduce_finish<FIN>(rp, acc);
    return;
  }
  DD accr[2] = {DD{0.0, 0.0}, DD{0.0, 0.0}}, acci[2] = {DD{0.0, 0.0}, DD{0.0, 0.0}};
  const Cx<R>* A = static_cast<const Cx<R>*>(p.b.base);
  const Cx<R>* B = static_cast<const Cx<R>*>(KIND == LD_NORM2 ? p.b.base : p.c.base);
  const bool pa = (KIND == LD_ADOT), pb = (KIND == LD_DOT_AA);
  int u = 0;
  for (SiteElemWalk w(d.ne); w.i < p.n; w.next(d.ne)) {
    const Cx<R>* a = A + w.i * d.ne;
    const Cx<R>* b = B + w.i * d.ne;
    const int pe = (pa || pb) ? perm_elem_n(d.perm, w.e, d.blk, d.inv_blk) : w.e;
    const Cx<R> ua = a[pa ? pe : w.e], vb = b[pb ? pe : w.e];
    const double ur = ua.re, ui = ua.im, vr = vb.re, vi = vb.im;
    double tr, ti = 0.0;
    if constexpr (KIND == LD_DOT || KIND == LD_REDOT || KIND == LD_NORM2) {
      tr = __dadd_rn(__dmul_rn(ur, vr), __dmul_rn(ui, vi));
      if constexpr (KIND == LD_DOT) ti = __dsub_rn(__dmul_rn(ur, vi), __dmul_rn(ui, vr));
    } else if constexpr (KIND == LD_DOT_AA) {
      tr = __dsub_rn(__dmul_rn(ur, vr), __dmul_rn(ui, vi));
      ti = __dsub_rn(__dmul_rn(-ur, vi), __dmul_rn(ui, vr));
    } else {
      tr = __dsub_rn(__dmul_rn(ur, vr), __dmul_rn(ui, vi));
      ti = __dadd_rn(__dmul_rn(ur, vi), __dmul_rn(ui, vr));
    }
    dd_add(accr[u], tr);
    if constexpr (FIN::NACC > 1) dd_add(acci[u], ti);
    u ^= 1;
  }
  DD acc[ArrN<FIN::NACC>::value];
  acc[0] = accr[0];
  dd_merge(acc[0], accr[1]);
  if constexpr (FIN::NACC > 1) {
    acc[1] = acci[0];
    dd_merge(acc[1], acci[1]);
  }
  reduce_finish<FIN>(rp, acc);
}

template <typename R, int KIND, typename OUT>
inline void api_gdot_n(const char* kid, int nc, int ne, int perm, void* r, Opnd a, Opnd b, const int* gang, int n) {
  constexpr int NACC = GDotFinish<KIND, OUT>::NACC;
  const size_t rbytes = NACC * sizeof(OUT);
  if (!nc_ok(kid, nc)) return;
  if (!r || (n > 0 && (!opnd_ok(a) || (KIND != LD_NORM2 && !opnd_ok(b))))) {
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
  const bool flat = gang == nullptr && a.mode == OM_CONTIG && (KIND == LD_NORM2 || b.mode == OM_CONTIG);
  long long grid = ((flat ? (long long)n * ne : (long long)n) + 255) / 256;
  const long long cap = (long long)sms * (flat ? 8 : 4);
  if (grid > cap) grid = cap;
  if (grid > rs->max_blocks) grid = rs->max_blocks;
  if (flat)
    gdotn_flat_kernel<R, KIND, OUT><<<(unsigned)(grid < 1 ? 1 : grid), 256, 0, st>>>(p, rp, nc_dims(nc, ne, perm));
  else
    gdotn_kernel<R, KIND, OUT><<<(unsigned)(grid < 1 ? 1 : grid), 256, 0, st>>>(p, rp, nc_dims(nc, ne, perm));
  if (!check_launch(kid)) return;
  if (!dev_out) {
    if (cudaMemcpyAsync(r, rs->result, rbytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      check_launch(kid);
  }
}

// global record sums with run-time record length NR (reals per record).
// Records whose lcm(NR, 32) fits a block use gsum_kernel's scheme (thread t
// of a block meets component t % NR on every step of a flat walk); larger
// records give each thread up to GSUM_Q components c = t + q * blockDim of
// every site, sites striding over the blocks.  Either way every component
// is added in double-double per thread, folded over the threads of a block
// in a fixed order into per-block partials, and over the blocks by
// gsum_fold_kernel (one block per component, a fixed order).
constexpr int GSUM_Q = 8;

template <typename R, bool WIDE>
__global__ void __launch_bounds__(1024, WIDE ? 1 : 2) gsumn_kernel(const EwParams p, int NR, DD* partials, int flat) {
  extern __shared__ __align__(16) unsigned char gsnm[];
  DD* red = reinterpret_cast<DD*>(gsnm);
  const int BT = blockDim.x;
  if constexpr (!WIDE) {
    const int c = threadIdx.x % NR;
    DD acc{0.0, 0.0};  // groups of GS_U loads summed by tree_sum, as gsum_kernel
    const long long total = p.n * NR;
    const long long stride = (long long)gridDim.x * BT;
    auto load = [&](long long j) -> double {
      if (flat) return (double)static_cast<const R*>(p.b.base)[j];
      const long long i = j / NR;
      const long long k = p.gang ? (long long)p.gang[i] : i;
      const R* rec = (p.b.mode == OM_PTR) ? static_cast<const R*>(p.b.ptrs[k]) : static_cast<const R*>(p.b.base) + k * NR;
      return (double)rec[c];
    };
    long long j = (long long)blockIdx.x * BT + threadIdx.x;
    for (; j + (GS_U - 1) * stride < total; j += GS_U * stride) {
      double v[GS_U];
#pragma unroll
      for (int u = 0; u < GS_U; u++) v[u] = load(j + u * stride);
      dd_add(acc, tree_sum(v));
    }
    for (; j < total; j += stride) dd_add(acc, load(j));
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int q = threadIdx.x; q < NR; q += BT) {
      DD s = red[q];
      for (int t = q + NR; t < BT; t += NR) dd_merge(s, red[t]);
      partials[(long long)blockIdx.x * NR + q] = s;
    }
  } else {
    DD acc[GSUM_Q];
#pragma unroll
    for (int q = 0; q < GSUM_Q; q++) acc[q] = DD{0.0, 0.0};
    for (long long i = blockIdx.x; i < p.n; i += gridDim.x) {
      const long long k = p.gang ? (long long)p.gang[i] : i;
      const R* rec = (p.b.mode == OM_PTR) ? static_cast<const R*>(p.b.ptrs[k]) : static_cast<const R*>(p.b.base) + k * NR;
#pragma unroll
      for (int q = 0; q < GSUM_Q; q++) {
        const int c = threadIdx.x + q * BT;
        if (c < NR) dd_add(acc[q], (double)rec[c]);
      }
    }
#pragma unroll
    for (int q = 0; q < GSUM_Q; q++) {
      const int c = threadIdx.x + q * BT;
      if (c < NR) partials[(long long)blockIdx.x * NR + c] = acc[q];
    }
  }
}

template <typename R, typename OUT = R>
inline void api_gsum_n(const char* kid, int nc, int ne, void* r, Opnd a, const int* gang, int n) {
  if (!nc_ok(kid, nc)) return;
  const int NR = 2 * ne;
  const size_t rbytes = (size_t)NR * sizeof(OUT);
  if (!r || (n > 0 && !opnd_ok(a))) {
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
  int l = NR;
  while (l % 32 && l <= 1024) l += NR;
  const int wide = (l > 1024) ? 1 : 0;
  int BT;
  if (!wide) {
    BT = l;
    while (BT + l <= 1024) BT += l;
  } else {
    BT = ((NR + GSUM_Q - 1) / GSUM_Q + 31) / 32 * 32;
    if (BT < 256) BT = 256;
    if (BT > 1024) {
      set_error(QLAGPU_ERR_ARG, kid, "record too large for the global sum (more than 16384 reals)");
      return;
    }
  }
  const int sms = device_sm_count();
  long long grid = wide ? (long long)n : ((long long)n * NR + BT - 1) / BT;
  const int per_sm = (wide ? 1024 : 2048) / BT;  // resident blocks (registers: 64 / 32 per thread)
  const long long cap = (long long)sms * (per_sm > 0 ? per_sm : 1);
  if (grid > cap) grid = cap;
  if (grid < 1) grid = 1;
  const long long need_ll = (grid * NR + ((long long)NR * (long long)sizeof(OUT) + (long long)sizeof(DD) - 1) /
                                            (long long)sizeof(DD) + 1) / 2 + 1;
  const int need = (int)need_ll;
  ReduceScratch* rs = reduce_scratch(st, need > 32 * sms + 64 ? need : 32 * sms + 64);
  if (!rs) return;
  OUT* res = dev_out ? static_cast<OUT*>(r) : reinterpret_cast<OUT*>(rs->partials + grid * NR);
  EwParams p;
  std::memset(&p, 0, sizeof(p));
  p.b = a;
  p.gang = gang;
  p.n = n;
  const int flat = (gang == nullptr && a.mode == OM_CONTIG) ? 1 : 0;
  const size_t smem = wide ? 0 : (size_t)BT * sizeof(DD);
  if (wide)
    gsumn_kernel<R, true><<<(unsigned)grid, BT, smem, st>>>(p, NR, rs->partials, flat);
  else
    gsumn_kernel<R, false><<<(unsigned)grid, BT, smem, st>>>(p, NR, rs->partials, flat);
  if (!check_launch(kid)) return;
  gsum_fold_kernel<OUT><<<NR, GS_FOLD, 0, st>>>(rs->partials, (int)grid, NR, res);
  if (!check_launch(kid)) return;
  if (!dev_out) {
    if (cudaMemcpyAsync(r, res, rbytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      check_launch(kid);
  }
}

// precision conversions with run-time record length
template <typename RIN, typename ROUT>
__global__ void __launch_bounds__(256) convertn_kernel(const EwParams p, int NR) {
  for (SiteElemWalk w(NR); w.i < p.n; w.next(NR)) {
    const long long k = p.gang ? (long long)p.gang[w.i] : w.i;
    const RIN* src = (p.b.mode == OM_PTR) ? static_cast<const RIN*>(p.b.ptrs[k]) : static_cast<const RIN*>(p.b.base) + k * NR;
    static_cast<ROUT*>(p.out)[k * NR + w.e] = static_cast<ROUT>(src[w.e]);
  }
}

template <typename RIN, typename ROUT>
inline void api_convert_n(const char* kid, int nc, int ne, void* r, Opnd a, const int* gang, int n) {
  if (!nc_ok(kid, nc) || n <= 0) return;
  if (!r || !opnd_ok(a)) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  EwParams p;
  std::memset(&p, 0, sizeof(p));
  p.out = r;
  p.b = a;
  p.gang = gang;
  p.n = n;
  convertn_kernel<RIN, ROUT><<<nc_grid((long long)n * 2 * ne), 256, 0, current_stream()>>>(p, 2 * ne);
  check_launch(kid);
}

// ---------------------------------------------------------------------------
// DiracPropagator products and the spin trace at nc colours
// (build_qla.pl:1588-1661, 942-968): one thread per output complex number,
// x = (peq | meq ? r : 0), then x (+|-)= a * b over k (kc, then ks), each
// product and sum rounded as the reference's QLA_c_{peq,meq}_*_times_* macros.
// e = ((ic*4 + is)*nc + jc)*4 + js for P, ic*nc + jc for the trace's M.
template <typename R, int KIND, bool CA, bool CB>
__global__ void __launch_bounds__(256) propn_kernel(const EwParams p, int nc) {
  const int nm = nc * nc, np = 16 * nc * nc;
  const int nel = (KIND == PK_TRACE) ? nm : np;
  const int ra = (KIND == PK_MP) ? nm : np, rb = (KIND == PK_PM) ? nm : np;
  const float inv_nc = 1.0f / (float)nc, inv_4nc = 1.0f / (float)(4 * nc);
  const bool minus = (p.eqop == MEQ || p.eqop == EQM), load = (p.eqop == PEQ || p.eqop == MEQ);
  auto pix = [nc](int i, int s, int j, int t, bool adj) {
    return adj ? ((j * 4 + t) * nc + i) * 4 + s : ((i * 4 + s) * nc + j) * 4 + t;
  };
  auto mix = [nc](int i, int j, bool adj) { return adj ? j * nc + i : i * nc + j; };
  for (SiteElemWalk w(nel); w.i < p.n; w.next(nel)) {
    const long long k = p.gang ? (long long)p.gang[w.i] : w.i;
    const Cx<R>* A = rec_ptr<R>(p.b, k, ra);
    Cx<R>* O = static_cast<Cx<R>*>(p.out) + k * nel + w.e;
    Cx<R> x = load ? *O : Cx<R>{R(0), R(0)};
    if constexpr (KIND == PK_TRACE) {
      const int ic = div_small(w.e, nc, inv_nc), jc = w.e - ic * nc;
      for (int s2 = 0; s2 < 4; s2++) {
        const Cx<R> v = A[pix(ic, s2, jc, s2, false)];
        x = minus ? Cx<R>{rsub(x.re, v.re), rsub(x.im, v.im)} : Cx<R>{radd(x.re, v.re), radd(x.im, v.im)};
      }
    } else {
      const Cx<R>* B = rec_ptr<R>(p.c, k, rb);
      const int row = div_small(w.e, 4 * nc, inv_4nc), col = w.e - row * 4 * nc;
      const int ic = row >> 2, is = row & 3, jc = col >> 2, js = col & 3;
      for (int kc = 0; kc < nc; kc++) {
        if constexpr (KIND == PK_PP) {
          for (int ks = 0; ks < 4; ks++) cmac<CA, CB>(x, minus, A[pix(ic, is, kc, ks, CA)], B[pix(kc, ks, jc, js, CB)]);
        } else if constexpr (KIND == PK_MP) {
          cmac<CA, CB>(x, minus, A[mix(ic, kc, CA)], B[pix(kc, is, jc, js, CB)]);
        } else {
          cmac<CA, CB>(x, minus, A[pix(ic, is, kc, js, CA)], B[mix(kc, jc, CB)]);
        }
      }
    }
    *O = x;
  }
}

template <typename R, int KIND, bool CA, bool CB>
inline void api_prop_n(const char* kid, int nc, void* r, Opnd a, Opnd b, const int* gang, int n, int eqop) {
  if (!nc_ok(kid, nc) || n <= 0) return;
  if (!r || !opnd_ok(a) || (KIND != PK_TRACE && !opnd_ok(b))) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL array argument");
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
  const long long nel = (KIND == PK_TRACE) ? (long long)nc * nc : 16LL * nc * nc;
  propn_kernel<R, KIND, CA, CB><<<nc_grid((long long)n * nel), 256, 0, current_stream()>>>(p, nc);
  check_launch(kid);
}

// ---------------------------------------------------------------------------
// multi-direction sums r (eqop) sum_d A_d b_d at nc colours (build_qla.pl:
// 1693-1727): one thread per (site, colour row); the row starts from 0
// (eq, eqm) or r (peq, meq) and takes every direction's products in the
// reference's order with the eqop's sign, each product and sum rounded.
struct MultiNParams {
  Opnd a[kMaxDirs], b[kMaxDirs];
  void* out;
  const int* gang;
  long long n;
  int nd, nc, minus, out_read;
};

template <typename R, bool ADJ>
__global__ void __launch_bounds__(256) multin_kernel(const MultiNParams p) {
  const int nc = p.nc;
  for (SiteElemWalk w(nc); w.i < p.n; w.next(nc)) {
    const long long k = p.gang ? (long long)p.gang[w.i] : w.i;
    const int ic = w.e;
    Cx<R>* out = static_cast<Cx<R>*>(p.out) + k * nc + ic;
    Cx<R> y = p.out_read ? *out : Cx<R>{R(0), R(0)};
    for (int d = 0; d < p.nd; d++) {
      const Cx<R>* A = rec_ptr<R>(p.a[d], k, nc * nc);
      const Cx<R>* B = rec_ptr<R>(p.b[d], k, nc);
      for (int kc = 0; kc < nc; kc++) cmac<ADJ, false>(y, p.minus != 0, A[ADJ ? kc * nc + ic : ic * nc + kc], B[kc]);
    }
    *out = y;
  }
}

template <typename R, bool ADJ>
inline void api_multi_n(const char* kid, int nc, void* r, const void* a, bool pa, const void* b, bool pb,
                        const int* gang, int n, int nd, int eqop) {
  if (!nc_ok(kid, nc) || n <= 0 || nd <= 0) return;
  if (!r || !a || !b) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  std::vector<const void*> av((size_t)nd), bv((size_t)nd);
  if (!multi_fetch_ptrs(a, nd, av.data()) || !multi_fetch_ptrs(b, nd, bv.data())) {
    check_launch(kid);
    return;
  }
  for (int d = 0; d < nd; d++)
    if (!av[(size_t)d] || !bv[(size_t)d]) {
      set_error(QLAGPU_ERR_NULLPTR, kid, "NULL direction operand");
      return;
    }
  for (int d0 = 0; d0 < nd; d0 += kMaxDirs) {
    MultiNParams p;
    std::memset(&p, 0, sizeof(p));
    p.nd = (nd - d0 < kMaxDirs) ? nd - d0 : kMaxDirs;
    p.nc = nc;
    p.out = r;
    p.gang = gang;
    p.n = n;
    p.minus = (eqop == MEQ || eqop == EQM) ? 1 : 0;
    p.out_read = (d0 > 0 || eqop == PEQ || eqop == MEQ) ? 1 : 0;
    for (int d = 0; d < p.nd; d++) {
      const void* ad = av[(size_t)(d0 + d)];
      const void* bd = bv[(size_t)(d0 + d)];
      p.a[d] = pa ? op_ptr(static_cast<const void* const*>(ad)) : op_contig(ad);
      p.b[d] = pb ? op_ptr(static_cast<const void* const*>(bd)) : op_contig(bd);
    }
    multin_kernel<R, ADJ><<<nc_grid((long long)n * nc), 256, 0, current_stream()>>>(p);
    if (!check_launch(kid)) return;
  }
}

}  // namespace qlab
