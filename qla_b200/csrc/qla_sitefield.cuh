// qla_sitefield.cuh -- the site-field families of the F3 / D3 level-1 API
// that fill, pick apart or re-arrange whole records, and the global
// reductions over records too large for one thread's registers:
//
//   X (eqop) x             one record broadcast to every site (v h d m p)
//   M (eqop) c             c times the identity at every site (diagfill)
//   X = zero;  X = a where mask != 0 (copymask)
//   C = elem(a, ...), elem(X, ...) = C, colour-column / Dirac-vector
//       extraction and insertion
//   D = gamma_mu D,  P = gamma_mu P,  P = P gamma_mu   (mu = 0..15)
//   C / R = trace, Re trace, Im trace of M;  M = traceless antihermitian part
//   c / r = global sums of Ma.M, P.P, P.Pa-type products, |P|^2
//   x = sum over sites of X (every component summed separately)
//
// Reference sections (lib/perl/build_qla.pl): constant fills :2584-2618,
// zero fills :2561-2582, copymask :2058-2084, array components :767-820,
// colour columns :822-876, Dirac vectors :878-931, trace :933-981,
// antihermitian part :983-1064, gamma multiplication :1358-1412 with the
// basis of lib/perl/expressions_gamma.pl:59-134, global inner products and
// norms :2089-2272, global sums :2449-2484.
//
// Element maps run one thread per output complex number, like the
// element-wise families: consecutive threads touch consecutive elements of
// the AoS records, which coalesces for every record size.  The gamma product
// on D and the antihermitian part run one site per thread on the site
// engine instead (GammaDOp, AntihermOp), which stages the records with bulk
// copies.  Every map here
// only moves values or negates / swaps components, except the trace and the
// antihermitian part, which repeat the reference's additions in its order;
// all results are bit-identical to the reference.
#pragma once
#include <cstdio>
#include "qla_ewise.cuh"

namespace qlab {

enum SfKind : int {
  SF_BCAST = 0,   // r (eqop) x                          (x one record)
  SF_DIAG,        // M r (eqop) c * identity
  SF_ZERO,        // r = 0
  SF_MASK,        // r = a where mask != 0
  SF_SUB,         // r.e[oi[j]] = a.e[si[j]], j < cnt    (components, columns)
  SF_GAMMA_L,     // r = gamma a   on the first spin index of P
  SF_GAMMA_R,     // r = a gamma   on the second spin index of P
  SF_TRACE_C,     // C r = trace a
  SF_TRACE_RE,    // R r = Re trace a
  SF_TRACE_IM,    // R r = Im trace a
  SF_ANTIHERM     // M r = traceless antihermitian part of a (N-colour maps; Nc = 3: AntihermOp)
};

struct SfParams {
  void* out;
  Opnd a;              // source field
  Opnd m;              // QLA_Int mask field (SF_MASK)
  const int* gang;
  long long n;
  int eqop;
  int cnt;             // SF_SUB: components copied per site
  int oi[12], si[12];  // SF_SUB: destination / source component of copy j
  int gs[4], gp[4];    // SF_GAMMA_*: source spin and phase (0: 1, 1: i, 2: -1, 3: -i) per destination spin
  const void* cptr;    // SF_BCAST / SF_DIAG: the constant in device memory, or nullptr (value in the argument)
};

// a record constant passed by value (kernel parameter space, read-only and
// broadcast to all threads)
template <typename R, int NE>
struct RecConst {
  Cx<R> v[NE];
};

// output complex numbers per site of each kind
template <int KIND, int NE_OUT>
struct SfOutPerSite {
  static constexpr int value = (KIND == SF_TRACE_C || KIND == SF_TRACE_RE || KIND == SF_TRACE_IM) ? 1 : NE_OUT;
};

template <typename R>
__device__ __forceinline__ Cx<R> phase_times(int ph, Cx<R> a) {
  // QLA_c_eq_c, QLA_c_eq_ic, QLA_c_eqm_c, QLA_c_eqm_ic (include/qla_complex.h:147-168)
  switch (ph) {
    case 0: return a;
    case 1: return Cx<R>{-a.im, a.re};
    case 2: return Cx<R>{-a.re, -a.im};
    default: return Cx<R>{a.im, -a.re};
  }
}

// NE_OUT / NE_SRC: complex numbers per destination / source record.
// For SF_GAMMA_* the record is a P (144); the spin index being multiplied
// is decoded from the element index below.
template <typename R, int NE_OUT, int NE_SRC, int KIND>
__global__ void __launch_bounds__(256) sf_kernel(const SfParams p, const RecConst<R, (KIND == SF_BCAST) ? NE_OUT : 1> cv) {
  constexpr int OPS = SfOutPerSite<KIND, NE_OUT>::value;
  const int ops = (KIND == SF_SUB) ? p.cnt : OPS;
  const long long total = p.n * ops;
  Cx<R> c1{R(0), R(0)};
  if constexpr (KIND == SF_DIAG) c1 = p.cptr ? *static_cast<const Cx<R>*>(p.cptr) : cv.v[0];
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const long long i = g / ops;
    const int e = (int)(g - i * ops);
    const long long k = p.gang ? (long long)p.gang[i] : i;
    if constexpr (KIND == SF_BCAST) {
      Cx<R>* out = static_cast<Cx<R>*>(p.out) + k * NE_OUT + e;
      const Cx<R> b = p.cptr ? static_cast<const Cx<R>*>(p.cptr)[e] : cv.v[e];
      const bool load = (p.eqop == PEQ || p.eqop == MEQ);
      const Cx<R> x = load ? *out : Cx<R>{R(0), R(0)};
      *out = ew_apply<R, EW_COPY>(p.eqop, x, Cx<R>{R(0), R(0)}, b, Cx<R>{R(0), R(0)});
    } else if constexpr (KIND == SF_DIAG) {
      // QLA_c_<eqop>_r(r_ij, 0.) on every element, then QLA_c_<eqop>_c(r_ii, c)
      // on the diagonal (build_qla.pl:2603-2616, make_code_unary.pl "diagfill")
      Cx<R>* out = static_cast<Cx<R>*>(p.out) + k * 9 + e;
      Cx<R> x;
      switch (p.eqop) {
        case EQ: x = Cx<R>{R(0), R(0)}; break;
        case EQM: x = Cx<R>{-R(0), R(0)}; break;
        case PEQ: x = *out; x.re = radd(x.re, R(0)); break;
        default: x = *out; x.re = rsub(x.re, R(0)); break;
      }
      if (e % 4 == 0) {
        switch (p.eqop) {
          case EQ: x = c1; break;
          case EQM: x = Cx<R>{-c1.re, -c1.im}; break;
          case PEQ: x = Cx<R>{radd(x.re, c1.re), radd(x.im, c1.im)}; break;
          default: x = Cx<R>{rsub(x.re, c1.re), rsub(x.im, c1.im)}; break;
        }
      }
      *out = x;
    } else if constexpr (KIND == SF_ZERO) {
      static_cast<Cx<R>*>(p.out)[k * NE_OUT + e] = Cx<R>{R(0), R(0)};
    } else if constexpr (KIND == SF_MASK) {
      const int mv = (p.m.mode == OM_PTR) ? *static_cast<const int*>(p.m.ptrs[k]) : static_cast<const int*>(p.m.base)[k];
      if (mv) static_cast<Cx<R>*>(p.out)[k * NE_OUT + e] = rec_ptr<R>(p.a, k, NE_SRC)[e];
    } else if constexpr (KIND == SF_SUB) {
      static_cast<Cx<R>*>(p.out)[k * NE_OUT + p.oi[e]] = rec_ptr<R>(p.a, k, NE_SRC)[p.si[e]];
    } else if constexpr (KIND == SF_GAMMA_L || KIND == SF_GAMMA_R) {
      // P: e = ((ic*4 + is)*3 + jc)*4 + js (D records take GammaDOp)
      int s, base, stride;
      if constexpr (KIND == SF_GAMMA_R) {
        s = e & 3;
        base = e - s;
        stride = 1;
      } else {
        s = (e / 12) & 3;
        base = e - s * 12;
        stride = 12;
      }
      const Cx<R> a = rec_ptr<R>(p.a, k, NE_SRC)[base + p.gs[s] * stride];
      static_cast<Cx<R>*>(p.out)[k * NE_OUT + e] = phase_times<R>(p.gp[s], a);
    } else if constexpr (KIND == SF_TRACE_C) {
      // QLA_c_eq_r(x, 0.); QLA_c_peq_c(x, a_ii) for i = 0, 1, 2 (build_qla.pl:933-981)
      const Cx<R>* a = rec_ptr<R>(p.a, k, 9);
      Cx<R> x{R(0), R(0)};
#pragma unroll
      for (int c = 0; c < 3; c++) x = Cx<R>{radd(x.re, a[c * 4].re), radd(x.im, a[c * 4].im)};
      static_cast<Cx<R>*>(p.out)[k] = x;
    } else if constexpr (KIND == SF_TRACE_RE || KIND == SF_TRACE_IM) {
      const Cx<R>* a = rec_ptr<R>(p.a, k, 9);
      R x = R(0);
#pragma unroll
      for (int c = 0; c < 3; c++) x = radd(x, KIND == SF_TRACE_RE ? a[c * 4].re : a[c * 4].im);
      static_cast<R*>(p.out)[k] = x;
    }
  }
}

template <typename R, int NE_OUT, int NE_SRC, int KIND>
inline void sf_launch(const char* kid, SfParams& p, const RecConst<R, (KIND == SF_BCAST) ? NE_OUT : 1>& cv) {
  const int ops = (KIND == SF_SUB) ? p.cnt : SfOutPerSite<KIND, NE_OUT>::value;
  const long long total = p.n * ops;
  const long long cap = (long long)device_sm_count() * 16;
  long long grid = (total + 255) / 256;
  if (grid > cap) grid = cap;
  sf_kernel<R, NE_OUT, NE_SRC, KIND><<<(unsigned)(grid < 1 ? 1 : grid), 256, 0, current_stream()>>>(p, cv);
  check_launch(kid);
}

inline bool sf_prep(const char* kid, SfParams& p, void* r, Opnd a, const int* gang, int n, int eqop, bool need_a) {
  if (n <= 0) return false;
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
  return true;
}

// X (eqop) x: x is one record, in host or device memory
template <typename R, int NE>
inline void api_fill(const char* kid, void* r, const void* x, const int* gang, int n, int eqop) {
  SfParams p;
  if (!sf_prep(kid, p, r, Opnd{}, gang, n, eqop, false)) return;
  if (!x) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  RecConst<R, NE> cv;
  if (is_device_ptr(x))
    p.cptr = x;
  else
    std::memcpy(&cv, x, sizeof(cv));
  sf_launch<R, NE, NE, SF_BCAST>(kid, p, cv);
}

// M (eqop) c * identity: c a complex number in host or device memory
template <typename R>
inline void api_diagfill(const char* kid, void* r, const void* c, const int* gang, int n, int eqop) {
  SfParams p;
  if (!sf_prep(kid, p, r, Opnd{}, gang, n, eqop, false)) return;
  if (!c) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  RecConst<R, 1> cv;
  if (is_device_ptr(c))
    p.cptr = c;
  else
    std::memcpy(&cv, c, sizeof(cv));
  sf_launch<R, 9, 9, SF_DIAG>(kid, p, cv);
}

template <typename R, int NE>
inline void api_zero(const char* kid, void* r, const int* gang, int n) {
  SfParams p;
  if (!sf_prep(kid, p, r, Opnd{}, gang, n, EQ, false)) return;
  sf_launch<R, NE, NE, SF_ZERO>(kid, p, RecConst<R, 1>{});
}

template <typename R, int NE>
inline void api_mask(const char* kid, void* r, Opnd a, Opnd m, const int* gang, int n) {
  SfParams p;
  if (!sf_prep(kid, p, r, a, gang, n, EQ, true)) return;
  if (!opnd_ok(m)) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  p.m = m;
  sf_launch<R, NE, NE, SF_MASK>(kid, p, RecConst<R, 1>{});
}

// component index of (ic, is, jc, js) in a record of the given type letter
// (include/qla_types.h:38-42: colour-major, spin inner)
inline int sf_elem(char t, int ic, int is, int jc, int js) {
  switch (t) {
    case 'V': return ic;
    case 'H': return ic * 2 + is;
    case 'D': return ic * 4 + is;
    case 'M': return ic * 3 + jc;
    case 'P': return ((ic * 4 + is) * 3 + jc) * 4 + js;
    default: return 0;  // 'C'
  }
}

// r.(DST component) = a.(SRC component) for every colour (and, for Dirac
// vectors, spin) index the function loops over.  WHAT selects the family:
//   'e' array component  (C <- X, X <- C; indices fixed by the arguments)
//   'c' colour column    (V <- H/D/M/P and back; the loop runs over ic)
//   'd' Dirac vector     (D <- P and back; the loop runs over ic, is)
template <typename R, int NE_OUT, int NE_SRC>
inline void api_sub(const char* kid, void* r, Opnd a, const int* gang, int n, char what, char dst, char src,
                    int i_c, int i_s, int j_c, int j_s) {
  SfParams p;
  if (!sf_prep(kid, p, r, a, gang, n, EQ, true)) return;
  // the container's fixed indices; the loop variable(s) fill the rest
  const char cont = (dst == 'V' || dst == 'C' || (what == 'd' && dst == 'D')) ? src : dst;
  // the reference does not check its indices; out-of-range ones would
  // address outside the records, so they are refused here
  if (i_c < 0 || i_c > 2 || i_s < 0 || i_s > (cont == 'H' ? 1 : 3) || j_c < 0 || j_c > 2 || j_s < 0 || j_s > 3) {
    set_error(QLAGPU_ERR_ARG, kid, "colour or spin index out of range");
    return;
  }
  int cnt = 0;
  auto put = [&](int ic, int is) {
    int o, s;
    if (what == 'e') {
      o = (dst == 'C') ? 0 : sf_elem(dst, i_c, i_s, j_c, j_s);
      s = (src == 'C') ? 0 : sf_elem(src, i_c, i_s, j_c, j_s);
    } else if (what == 'c') {
      // the colour loop index is ic; in an M the column vector is (ic, j_c)
      const int ce = sf_elem(cont, ic, i_s, j_c, j_s);
      o = (dst == 'V') ? ic : ce;
      s = (src == 'V') ? ic : ce;
    } else {
      const int pe = sf_elem('P', ic, is, j_c, j_s);
      const int de = sf_elem('D', ic, is, 0, 0);
      o = (dst == 'D') ? de : pe;
      s = (src == 'D') ? de : pe;
    }
    p.oi[cnt] = o;
    p.si[cnt] = s;
    cnt++;
  };
  if (what == 'e') {
    put(0, 0);
  } else if (what == 'c') {
    for (int ic = 0; ic < 3; ic++) put(ic, 0);
  } else {
    for (int ic = 0; ic < 3; ic++)
      for (int is = 0; is < 4; is++) put(ic, is);
  }
  p.cnt = cnt;
  sf_launch<R, NE_OUT, NE_SRC, SF_SUB>(kid, p, RecConst<R, 1>{});
}

// gamma_mu = product of the basis matrices gamma_b for the set bits b of mu,
// in increasing bit order (lib/perl/expressions_gamma.pl:59-134, the
// DeGrand-Rossi basis).  Every row and column holds exactly one entry from
// {1, i, -1, -i}.  Entries are (re, im) pairs of small integers.
struct GammaTable {
  int row_src[16][4], row_ph[16][4];  // left:  r_s = ph * a_src (row s of gamma)
  int col_src[16][4], col_ph[16][4];  // right: r_s = ph * a_src (column s of gamma)
};

inline const GammaTable& gamma_table() {
  static const GammaTable tab = [] {
    // basis gamma_x, gamma_y, gamma_z, gamma_t as (re, im) per entry [row][col]
    static const int G[4][4][4][2] = {
        {{{0, 0}, {0, 0}, {0, 0}, {0, 1}},
         {{0, 0}, {0, 0}, {0, 1}, {0, 0}},
         {{0, 0}, {0, -1}, {0, 0}, {0, 0}},
         {{0, -1}, {0, 0}, {0, 0}, {0, 0}}},
        {{{0, 0}, {0, 0}, {0, 0}, {-1, 0}},
         {{0, 0}, {0, 0}, {1, 0}, {0, 0}},
         {{0, 0}, {1, 0}, {0, 0}, {0, 0}},
         {{-1, 0}, {0, 0}, {0, 0}, {0, 0}}},
        {{{0, 0}, {0, 0}, {0, 1}, {0, 0}},
         {{0, 0}, {0, 0}, {0, 0}, {0, -1}},
         {{0, -1}, {0, 0}, {0, 0}, {0, 0}},
         {{0, 0}, {0, 1}, {0, 0}, {0, 0}}},
        {{{0, 0}, {0, 0}, {1, 0}, {0, 0}},
         {{0, 0}, {0, 0}, {0, 0}, {1, 0}},
         {{1, 0}, {0, 0}, {0, 0}, {0, 0}},
         {{0, 0}, {1, 0}, {0, 0}, {0, 0}}}};
    GammaTable t{};
    for (int mu = 0; mu < 16; mu++) {
      int m[4][4][2] = {};
      for (int d = 0; d < 4; d++) m[d][d][0] = 1;
      for (int b = 0; b < 4; b++) {
        if (!(mu & (1 << b))) continue;
        int q[4][4][2] = {};
        for (int r = 0; r < 4; r++)
          for (int c = 0; c < 4; c++)
            for (int x = 0; x < 4; x++) {
              q[r][c][0] += m[r][x][0] * G[b][x][c][0] - m[r][x][1] * G[b][x][c][1];
              q[r][c][1] += m[r][x][0] * G[b][x][c][1] + m[r][x][1] * G[b][x][c][0];
            }
        std::memcpy(m, q, sizeof(m));
      }
      auto ph = [](const int* v) { return v[0] == 1 ? 0 : v[1] == 1 ? 1 : v[0] == -1 ? 2 : 3; };
      for (int s = 0; s < 4; s++)
        for (int x = 0; x < 4; x++) {
          if (m[s][x][0] || m[s][x][1]) {
            t.row_src[mu][s] = x;
            t.row_ph[mu][s] = ph(m[s][x]);
          }
          if (m[x][s][0] || m[x][s][1]) {
            t.col_src[mu][s] = x;
            t.col_ph[mu][s] = ph(m[x][s]);
          }
        }
    }
    return t;
  }();
  return tab;
}

// D = gamma_mu D through the site engine: one site per thread, the record
// staged by the engine's bulk copies.  aux packs, per destination spin s,
// the source spin (bits 4s..4s+1) and the phase (bits 4s+2..4s+3).
template <typename R_>
struct GammaDOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = 12, N1 = 0, N2 = 0, NOUT = 12, NACC = 0;
  __device__ __forceinline__ static void apply(const SiteParams& p, const Cx<R> (&a)[N0], const Cx<R> (&)[1],
                                               const Cx<R> (&)[1], Cx<R> (&y)[NOUT]) {
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const int src = (p.aux >> (4 * s)) & 3, ph = (p.aux >> (4 * s + 2)) & 3;
#pragma unroll
      for (int ic = 0; ic < 3; ic++) {
        const Cx<R> v = src == 0 ? a[ic * 4] : src == 1 ? a[ic * 4 + 1] : src == 2 ? a[ic * 4 + 2] : a[ic * 4 + 3];
        y[ic * 4 + s] = phase_times<R>(ph, v);
      }
    }
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// M = traceless antihermitian part of M through the site engine
// (build_qla.pl:983-1064: x = sum Im a_cc / 3, r_ii = i (Im a_ii - x);
// x2 = (a_ij - conj(a_ji)) 0.5 for i < j, r_ij = x2, r_ji = -conj(x2))
template <typename R_>
struct AntihermOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = 9, N1 = 0, N2 = 0, NOUT = 9, NACC = 0;
  __device__ __forceinline__ static void apply(const SiteParams&, const Cx<R> (&a)[N0], const Cx<R> (&)[1],
                                               const Cx<R> (&)[1], Cx<R> (&y)[NOUT]) {
    R x = R(0);
#pragma unroll
    for (int c = 0; c < 3; c++) x = radd(x, a[c * 4].im);
    x = rdiv(x, R(3));
#pragma unroll
    for (int c = 0; c < 3; c++) y[c * 4] = Cx<R>{R(0), rsub(a[c * 4].im, x)};
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = i + 1; j < 3; j++) {
        const Cx<R> u = a[i * 3 + j], v = a[j * 3 + i];
        const Cx<R> x2{rmul(rsub(u.re, v.re), R(0.5)), rmul(radd(u.im, v.im), R(0.5))};
        y[i * 3 + j] = x2;
        y[j * 3 + i] = Cx<R>{-x2.re, x2.im};
      }
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// D = gamma_mu D, P = gamma_mu P (LEFT) or P = P gamma_mu
template <typename R, int NE, bool LEFT>
inline void api_gamma(const char* kid, void* r, Opnd a, int mu, const int* gang, int n) {
  if (mu < 0 || mu > 15) {
    // the reference prints this and leaves r unchanged (expressions_gamma.pl:466-470)
    std::printf("Gamma matrix %d not supported\n", mu);
    set_error(QLAGPU_ERR_ARG, kid, "gamma matrix index outside 0..15");
    return;
  }
  const GammaTable& t = gamma_table();
  if constexpr (NE == 12 && LEFT) {
    if (n <= 0) return;
    if (!r || !opnd_ok(a)) {
      set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
      return;
    }
    SiteParams sp = make_params(n, EQ);
    sp.in[0] = a;
    sp.out = r;
    sp.gang = gang;
    for (int s = 0; s < 4; s++) sp.aux |= (t.row_src[mu][s] | (t.row_ph[mu][s] << 2)) << (4 * s);
    SiteLauncher<GammaDOp<R>>::run(sp, kid);
  } else {
    SfParams p;
    if (!sf_prep(kid, p, r, a, gang, n, EQ, true)) return;
    for (int s = 0; s < 4; s++) {
      p.gs[s] = LEFT ? t.row_src[mu][s] : t.col_src[mu][s];
      p.gp[s] = LEFT ? t.row_ph[mu][s] : t.col_ph[mu][s];
    }
    if constexpr (LEFT)
      sf_launch<R, NE, NE, SF_GAMMA_L>(kid, p, RecConst<R, 1>{});
    else
      sf_launch<R, NE, NE, SF_GAMMA_R>(kid, p, RecConst<R, 1>{});
  }
}

template <typename R, int KIND>
inline void api_trace(const char* kid, void* r, Opnd a, const int* gang, int n) {
  SfParams p;
  if (!sf_prep(kid, p, r, a, gang, n, EQ, true)) return;
  sf_launch<R, 1, 9, KIND>(kid, p, RecConst<R, 1>{});
}

template <typename R>
inline void api_antiherm(const char* kid, void* r, Opnd a, const int* gang, int n) {
  api_map<AntihermOp<R>>(kid, r, a, Opnd{}, gang, n, EQ);
}

// ---------------------------------------------------------------------------
// Global reductions over P records and over the permuted (Ma, Pa) forms:
// every term is formed in double as the reference forms it and added in
// double-double.  Contiguous fields stream as one flat array of complex
// numbers (gdot_flat_kernel); gang-indexed or pointer-array fields take one
// thread per site (gdot_kernel).

template <int KIND, typename OUT>
struct GDotFinish {
  static constexpr int NACC = (KIND >= LD_REDOT) ? 1 : 2;
  __device__ static void finish(const SiteParams& p, const double* tot) {
    if constexpr (NACC == 1)
      write_real<OUT>(p, tot[0]);
    else
      write_cplx<OUT>(p, tot[0], tot[1]);
  }
};

// one complex term of the global sum, as ldot_site forms it, for element e
// of the site whose records start at a / b
template <typename R, int NE, int KIND, int PERM>
__device__ __forceinline__ void gdot_term(const Cx<R>* a, const Cx<R>* b, int e, double& tr, double& ti) {
  Cx<R> ua = a[e], vb = b[e];
  if constexpr (KIND == LD_ADOT) ua = a[perm_elem<PERM, NE>(e)];
  if constexpr (KIND == LD_DOT_AA) vb = b[perm_elem<PERM, NE>(e)];
  const double ur = ua.re, ui = ua.im, vr = vb.re, vi = vb.im;
  ti = 0.0;
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
}

// GS_U loads of one component in flight per thread, summed in double by
// tree_sum, then one double-double add per group: one accumulator keeps the
// registers low enough for two blocks of up to 1024 threads per SM.
constexpr int GS_U = 8;

// Contiguous operands without a gang index: the n * NE complex elements are
// one flat stream; thread g takes elements g, g + stride, ..., GD_U of them
// in flight, whose terms are summed in double by a fixed tree and then added
// in double-double; then the block / grid fold of reduce_finish.  The order
// of the sum differs from the reference's single running double (the global
// sums are compared to it within the stated tolerance); every term is formed
// in double exactly as the reference forms it.  Element positions are only
// decoded (a 64-bit division by NE) for the permuted (adjoint) forms.
constexpr int GD_U = 8;

template <typename R, int NE, int KIND, int PERM, typename OUT>
__global__ void __launch_bounds__(256, 4) gdot_flat_kernel(const EwParams p, const SiteParams rp) {
  using FIN = GDotFinish<KIND, OUT>;
  constexpr bool PLAIN = (KIND == LD_DOT || KIND == LD_REDOT || KIND == LD_NORM2);
  DD acc[ArrN<FIN::NACC>::value];
#pragma unroll
  for (int a = 0; a < ArrN<FIN::NACC>::value; a++) acc[a] = DD{0.0, 0.0};
  const Cx<R>* A = static_cast<const Cx<R>*>(p.b.base);
  const Cx<R>* B = static_cast<const Cx<R>*>(KIND == LD_NORM2 ? p.b.base : p.c.base);
  const long long total = p.n * NE;
  const long long stride = (long long)gridDim.x * blockDim.x;
  auto term = [&](long long q, double& tr, double& ti) {
    if constexpr (PLAIN) {
      gdot_term<R, NE, KIND, PERM>(A + q, B + q, 0, tr, ti);
    } else {
      const long long i = q / NE;
      const int e = (int)(q - i * NE);
      gdot_term<R, NE, KIND, PERM>(A + i * NE, B + i * NE, e, tr, ti);
    }
  };
  long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; g + (GD_U - 1) * stride < total; g += GD_U * stride) {
    double tr[GD_U], ti[GD_U];
#pragma unroll
    for (int u = 0; u < GD_U; u++) term(g + u * stride, tr[u], ti[u]);
    dd_add(acc[0], tree_sum(tr));
    if constexpr (FIN::NACC > 1) dd_add(acc[1], tree_sum(ti));
  }
  for (; g < total; g += stride) {
    double tr, ti;
    term(g, tr, ti);
    dd_add(acc[0], tr);
    if constexpr (FIN::NACC > 1) dd_add(acc[1], ti);
  }
  reduce_finish<FIN>(rp, acc);
}

// gang-indexed or pointer-array operands: one thread per site, the site's
// sum formed in double in the reference's element order (ldot_site)
template <typename R, int NE, int KIND, int PERM, typename OUT>
__global__ void __launch_bounds__(128) gdot_kernel(const EwParams p, const SiteParams rp) {
  using FIN = GDotFinish<KIND, OUT>;
  DD acc[ArrN<FIN::NACC>::value];
#pragma unroll
  for (int a = 0; a < ArrN<FIN::NACC>::value; a++) acc[a] = DD{0.0, 0.0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < p.n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long k = p.gang ? (long long)p.gang[i] : i;
    const Cx<R>* a = rec_ptr<R>(p.b, k, NE);
    const Cx<R>* b = (KIND == LD_NORM2) ? a : rec_ptr<R>(p.c, k, NE);
    double xr, xi;
    ldot_site<R, NE, KIND, PERM>(a, b, xr, xi);
    dd_add(acc[0], xr);
    if constexpr (FIN::NACC > 1) dd_add(acc[1], xi);
  }
  reduce_finish<FIN>(rp, acc);
}

// r: host (synchronous) or device (asynchronous) output of OUT values
template <typename R, int NE, int KIND, int PERM, typename OUT>
inline void api_gdot(const char* kid, void* r, Opnd a, Opnd b, const int* gang, int n) {
  constexpr int NACC = GDotFinish<KIND, OUT>::NACC;
  const size_t rbytes = NACC * sizeof(OUT);
  if (!r || (n > 0 && (!opnd_ok(a) || (KIND != LD_NORM2 && !opnd_ok(b))))) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  cudaStream_t st = current_stream();
  const bool dev_out = is_device_ptr(r);
  if (n <= 0) {
    // the reference loops zero times and stores its zero sum
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
  if (flat) {
    long long grid = ((long long)n * NE + 256 * GD_U - 1) / (256 * GD_U);
    const long long cap = (long long)sms * 8;
    if (grid > cap) grid = cap;
    if (grid > rs->max_blocks) grid = rs->max_blocks;
    gdot_flat_kernel<R, NE, KIND, PERM, OUT><<<(unsigned)(grid < 1 ? 1 : grid), 256, 0, st>>>(p, rp);
  } else {
    long long grid = ((long long)n + 127) / 128;
    const long long cap = (long long)sms * 8;
    if (grid > cap) grid = cap;
    if (grid > rs->max_blocks) grid = rs->max_blocks;
    gdot_kernel<R, NE, KIND, PERM, OUT><<<(unsigned)(grid < 1 ? 1 : grid), 128, 0, st>>>(p, rp);
  }
  if (!check_launch(kid)) return;
  if (!dev_out) {
    if (cudaMemcpyAsync(r, rs->result, rbytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      check_launch(kid);
  }
}

// ---------------------------------------------------------------------------
// Global record sums x = sum_i a[i] (build_qla.pl:2449-2484): every real
// component is summed over the sites separately.  A block of BT threads (a
// multiple of the NR reals per record and of 32) reads the records as one
// flat stream, so thread t always meets component t % NR and the loads are
// coalesced; each thread adds groups of GS_U loads in double-double and the
// block folds the threads of each component in a fixed order into
// per-block partials.  A
// second launch (gsum_fold_kernel, one block per component) folds the
// partials: thread t takes blocks t, t + 128, ... in order, then a fixed
// shared-memory tree.  For P records (NR = 288) the partials are megabytes,
// which one block folding them serially would take longer to read than the
// field itself.

template <typename R, int NR>
__global__ void __launch_bounds__(1024, 2) gsum_kernel(const EwParams p, DD* partials, int flat) {
  extern __shared__ __align__(16) unsigned char gssm[];
  DD* red = reinterpret_cast<DD*>(gssm);
  const int BT = blockDim.x;
  const int c = threadIdx.x % NR;
  DD acc{0.0, 0.0};
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
}

constexpr int GS_FOLD = 128;

template <typename OUT>
__global__ void __launch_bounds__(GS_FOLD) gsum_fold_kernel(const DD* __restrict__ partials, int nblk, int nr,
                                                            OUT* result) {
  __shared__ DD red[GS_FOLD];
  const int q = blockIdx.x;
  DD s{0.0, 0.0};
  for (int b = threadIdx.x; b < nblk; b += GS_FOLD) dd_merge(s, partials[(long long)b * nr + q]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = GS_FOLD / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) dd_merge(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) result[q] = static_cast<OUT>(__dadd_rn(red[0].hi, red[0].lo));
}

// r: one record of OUT components (host: synchronous, device: asynchronous)
template <typename R, int NE, typename OUT = R>
inline void api_gsum(const char* kid, void* r, Opnd a, const int* gang, int n) {
  constexpr int NR = 2 * NE;
  const size_t rbytes = NR * sizeof(OUT);
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
  // block: a multiple of lcm(NR, 32) reals, up to 1024 threads; one wave of
  // blocks (2048 resident threads per SM)
  int l = NR;
  while (l % 32) l += NR;
  int BT = l;
  while (BT + l <= 1024) BT += l;
  const int sms = device_sm_count();
  long long grid = ((long long)n * NR + BT - 1) / BT;
  const long long cap = (long long)sms * (2048 / BT > 0 ? 2048 / BT : 1);
  if (grid > cap) grid = cap;
  if (grid < 1) grid = 1;
  // partials [grid * NR] DD, then the result record
  const int need = (int)((grid * NR + (NR * sizeof(OUT) + sizeof(DD) - 1) / sizeof(DD) + 1) / 2 + 1);
  ReduceScratch* rs = reduce_scratch(st, need > 32 * sms + 64 ? need : 32 * sms + 64);
  if (!rs) return;
  DD* partials = rs->partials;
  OUT* res = dev_out ? static_cast<OUT*>(r) : reinterpret_cast<OUT*>(rs->partials + grid * NR);
  EwParams p;
  std::memset(&p, 0, sizeof(p));
  p.b = a;
  p.gang = gang;
  p.n = n;
  const int flat = (gang == nullptr && a.mode == OM_CONTIG) ? 1 : 0;
  gsum_kernel<R, NR><<<(unsigned)grid, BT, (size_t)BT * sizeof(DD), st>>>(p, partials, flat);
  if (!check_launch(kid)) return;
  gsum_fold_kernel<OUT><<<NR, GS_FOLD, 0, st>>>(partials, (int)grid, NR, res);
  if (!check_launch(kid)) return;
  if (!dev_out) {
    if (cudaMemcpyAsync(r, res, rbytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      check_launch(kid);
  }
}

// ---------------------------------------------------------------------------
// Precision conversions X_D <- X_F (QLA_DF3_X_*eq_X: exact promotion) and
// X_F <- X_D (QLA_FD3_X_*eq_X: one round-to-nearest per component),
// build_qla.pl:356-400 with QLA_DF_c_eq_c / QLA_FD_c_eq_c
// (include/qla_complex.h): one thread per real component.
template <typename RIN, typename ROUT, int NR>
__global__ void __launch_bounds__(256) convert_kernel(const EwParams p) {
  const long long total = p.n * NR;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const long long i = g / NR;
    const int c = (int)(g - i * NR);
    const long long k = p.gang ? (long long)p.gang[i] : i;
    const RIN* src = (p.b.mode == OM_PTR) ? static_cast<const RIN*>(p.b.ptrs[k]) : static_cast<const RIN*>(p.b.base) + k * NR;
    static_cast<ROUT*>(p.out)[k * NR + c] = static_cast<ROUT>(src[c]);
  }
}

template <typename RIN, typename ROUT, int NE>
inline void api_convert(const char* kid, void* r, Opnd a, const int* gang, int n) {
  if (n <= 0) return;
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
  const long long total = (long long)n * 2 * NE;
  const long long cap = (long long)device_sm_count() * 16;
  long long grid = (total + 255) / 256;
  if (grid > cap) grid = cap;
  convert_kernel<RIN, ROUT, 2 * NE><<<(unsigned)(grid < 1 ? 1 : grid), 256, 0, current_stream()>>>(p);
  check_launch(kid);
}

}  // namespace qlab
