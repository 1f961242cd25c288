// qla_prop.cuh -- DiracPropagator (P = [nc][4][nc][4] complex, 1152 B in F3)
// products and spin trace:
//   P (eqop) A * P'   A a colour matrix (or its adjoint), P' = P or P^+
//   P (eqop) P' * A
//   P (eqop) P' * P''  (12 x 12 spin-colour matrix product)
//   M (eqop) spintrace(P)
// (lib/perl/build_qla.pl:1588-1622 left multiplication, :1627-1661 right
// multiplication, expressions_tensor.pl:766; spin trace build_qla.pl:942-968).
//
// A P record does not fit in registers, and one thread per site would read it
// with a 1152-B stride.  Instead one thread computes ONE output element of one
// site: consecutive threads produce consecutive elements, so the operand
// elements they read (P'[..][jc][js] for fixed k) and the results they write
// are contiguous in memory -- coalesced AoS access without staging -- and the
// matrix / row operands shared by the 144 threads of a site come from L1.
// Every output element is accumulated exactly as the reference does (x = 0 or
// r, then x (+|-)= a*b over k in order), so results are bit-identical.
#pragma once
#include "qla_launch.cuh"
#include "qla_ops.cuh"

namespace qlab {

enum PKind : int { PK_MP = 0, PK_PM = 1, PK_PP = 2, PK_TRACE = 3 };

struct PropParams {
  Opnd a, b;
  void* out;
  const int* gang;
  long long n;
  int eqop;
};

template <typename R>
__device__ __forceinline__ Cx<R> ld_elem(const Opnd& o, long long k, int e, int rec) {
  const Cx<R>* base;
  if (o.mode == OM_PTR)
    base = static_cast<const Cx<R>*>(o.ptrs[k]);
  else
    base = static_cast<const Cx<R>*>(o.base) + k * rec;
  return base[e];
}

// element (i, s, j, t) of P or of P^+ (P^+[i][s][j][t] = conj P[j][t][i][s])
__device__ __forceinline__ int p_idx(int i, int s, int j, int t, bool adj) {
  return adj ? ((j * 4 + t) * 3 + i) * 4 + s : ((i * 4 + s) * 3 + j) * 4 + t;
}
__device__ __forceinline__ int m_idx(int i, int j, bool adj) { return adj ? j * 3 + i : i * 3 + j; }

template <typename R, int KIND, bool CA, bool CB>
__global__ void __launch_bounds__(256) prop_kernel(const PropParams p) {
  constexpr int NEL = (KIND == PK_TRACE) ? 9 : 144;  // output elements per site
  constexpr int RP = 144, RM = 9;
  const long long total = p.n * NEL;
  const bool minus = (p.eqop == MEQ || p.eqop == EQM);
  const bool load = (p.eqop == PEQ || p.eqop == MEQ);
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const long long i = g / NEL;
    const int e = (int)(g - i * NEL);
    const long long k = p.gang ? (long long)p.gang[i] : i;
    Cx<R>* out = static_cast<Cx<R>*>(p.out) + k * NEL + e;
    Cx<R> x = load ? *out : Cx<R>{R(0), R(0)};
    if constexpr (KIND == PK_TRACE) {
      const int ic = e / 3, jc = e % 3;
#pragma unroll
      for (int s = 0; s < 4; s++) {
        const Cx<R> v = ld_elem<R>(p.a, k, ((ic * 4 + s) * 3 + jc) * 4 + s, RP);
        if (minus) {
          x.re = rsub(x.re, v.re);
          x.im = rsub(x.im, v.im);
        } else {
          x.re = radd(x.re, v.re);
          x.im = radd(x.im, v.im);
        }
      }
    } else {
      const int ic = e / 48, is = (e / 12) % 4, jc = (e / 4) % 3, js = e % 4;
      if constexpr (KIND == PK_MP) {
#pragma unroll
        for (int kc = 0; kc < 3; kc++)
          cmac<CA, CB>(x, minus, ld_elem<R>(p.a, k, m_idx(ic, kc, CA), RM),
                       ld_elem<R>(p.b, k, p_idx(kc, is, jc, js, CB), RP));
      } else if constexpr (KIND == PK_PM) {
#pragma unroll
        for (int kc = 0; kc < 3; kc++)
          cmac<CA, CB>(x, minus, ld_elem<R>(p.a, k, p_idx(ic, is, kc, js, CA), RP),
                       ld_elem<R>(p.b, k, m_idx(kc, jc, CB), RM));
      } else {
#pragma unroll
        for (int kc = 0; kc < 3; kc++)
#pragma unroll
          for (int ks = 0; ks < 4; ks++)
            cmac<CA, CB>(x, minus, ld_elem<R>(p.a, k, p_idx(ic, is, kc, ks, CA), RP),
                         ld_elem<R>(p.b, k, p_idx(kc, ks, jc, js, CB), RP));
      }
    }
    *out = x;
  }
}

template <typename R, int KIND, bool CA, bool CB>
inline void api_prop(const char* kid, void* r, Opnd a, Opnd b, const int* gang, int n, int eqop) {
  if (n <= 0) return;
  if (!r || !opnd_ok(a) || (KIND != PK_TRACE && !opnd_ok(b))) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL array argument");
    return;
  }
  PropParams p;
  std::memset(&p, 0, sizeof(p));
  p.a = a;
  p.b = b;
  p.out = r;
  p.gang = gang;
  p.n = n;
  p.eqop = eqop;
  const long long total = (long long)n * ((KIND == PK_TRACE) ? 9 : 144);
  long long grid = (total + 255) / 256;
  const long long cap = (long long)device_sm_count() * 16;
  if (grid > cap) grid = cap;
  prop_kernel<R, KIND, CA, CB><<<(unsigned)(grid < 1 ? 1 : grid), 256, 0, current_stream()>>>(p);
  check_launch(kid);
}

}  // namespace qlab
