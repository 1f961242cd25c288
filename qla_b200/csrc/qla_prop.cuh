// qla_prop.cuh -- DiracPropagator (P = [nc][4][nc][4] complex, 1152 B in F3)
// products and spin trace:
//   P (eqop) A * P'   A a colour matrix (or its adjoint), P' = P or P^+
//   P (eqop) P' * A
//   P (eqop) P' * P''  (12 x 12 spin-colour matrix product)
//   M (eqop) spintrace(P)
// (lib/perl/build_qla.pl:1588-1622 left multiplication, :1627-1661 right
// multiplication, expressions_tensor.pl:766; spin trace build_qla.pl:942-968).
//
// A P record does not fit in one thread's registers, so several threads share
// a site.  Contiguous, 16-B aligned operands without a gang index go through
// one bulk-copy (TMA) pipeline of 8-site tiles (prop_tma_kernel: a producer
// warp stages the tile's records, the consumer threads compute from shared
// memory):
//   M * P   24 threads per site, thread (is, jc, jh) accumulates outputs
//           (ic, is, jc, 2jh..2jh+1) over ic;
//   P * M   24 threads per site, thread (ic, is, jh) accumulates outputs
//           (ic, is, jc, 2jh..2jh+1) over jc;
//   P * P   F3 12 threads per site, 2 output rows x 6 columns each in packed
//           FP32x2 arithmetic; D3 24 threads per site, one row x 6 columns.
// Gang, pointer or unaligned operands (and the last n mod 8 sites of M * P
// and P * M) run direct kernels that read every operand element once, in
// 16-B (F3) / 32-B (D3) runs of two consecutive complex numbers, consecutive
// threads touching consecutive runs:
//   M * P   24 threads per site, thread (is, jc, js pair): the P run
//           P[kc][is][jc][js..js+1] serves all three output colours ic;
//   P * M   24 threads per site, thread (ic, is, js pair): the P run
//           P[ic][is][kc][js..js+1] serves all three output colours jc;
//   P * P   6 (F3) / 12 (D3) threads per site, a column block of the second
//           operand in registers (prop_pp_kernel);
// there the 9 matrix elements come from L1 (shared by a site's threads), and
// adjoint or pointer operands are read element by element.  Every output
// element is accumulated exactly as the reference does (x = 0 or r, then
// x (+|-)= a*b over k in order), so results are bit-identical.  The spin
// trace keeps one thread per output element (9 per site).
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
  int vec_a, vec_b, vec_out;  // 16-B vector access allowed (contiguous, aligned)
  float negzero;              // -0.0f, passed at run time (see f2_mul)
  unsigned* err;              // device error word (bounded waits of the bulk-copy P * P)
  int stages;                 // stage ring depth of the bulk-copy P * P
};

// ---------------------------------------------------------------------------
// Packed FP32x2 arithmetic with per-lane rounding identical to the scalar
// __fmul_rn / __fadd_rn / __fsub_rn.  A pair of floats lives in one 64-bit
// register (F2: low lane first), so that a chain of packed operations needs
// no packing between them.  The packed add and sub are used as they are.  A
// packed product followed by a packed add is fused into one multiply-add by
// the compiler even with explicit .rn rounding (measured on sm_100a: every
// result equal to fmaf, none to the separately rounded pair), so the product
// is written as fma(a, b, z) with z = (-0, -0): a*b + (-0) rounds exactly as
// a*b alone, signed zeros included, and because z comes from a kernel
// argument the compiler cannot fold it into a plain product again.
using F2 = unsigned long long;
__device__ __forceinline__ F2 f2_pack(float lo, float hi) {
  F2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ float f2_lo(F2 v) { return __uint_as_float((unsigned)v); }
__device__ __forceinline__ float f2_hi(F2 v) { return __uint_as_float((unsigned)(v >> 32)); }
__device__ __forceinline__ F2 f2_neg(F2 v) { return v ^ 0x8000000080000000ull; }  // both lanes, exactly
__device__ __forceinline__ F2 f2_mul(F2 a, F2 b, F2 z) {
  F2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(z));
  return r;
}
__device__ __forceinline__ F2 f2_add(F2 a, F2 b) {
  F2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ F2 f2_sub(F2 a, F2 b) {
  F2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}

// x (+|-)= a * b for two output columns at once: lanes hold columns j0, j1
// (b's real parts bre, imaginary parts bim), a is broadcast (ar = (a.re,
// a.re), ai = (a.im, a.im)).  Per lane the operations and their order are
// cmac<CA, CB>'s.
template <bool CA, bool CB>
__device__ __forceinline__ void cmac_f2(F2& xre, F2& xim, bool minus, F2 ar, F2 ai, F2 bre, F2 bim, F2 z) {
  const F2 p1 = f2_mul(ar, bre, z), p2 = f2_mul(ai, bim, z);
  const F2 p3 = f2_mul(ar, bim, z), p4 = f2_mul(ai, bre, z);
  F2 re, im;
  if constexpr (!CA && !CB) {
    re = f2_sub(p1, p2);
    im = f2_add(p3, p4);
  } else if constexpr (CA && !CB) {
    re = f2_add(p1, p2);
    im = f2_sub(p3, p4);
  } else if constexpr (!CA && CB) {
    re = f2_add(p1, p2);
    im = f2_sub(p4, p3);
  } else {
    re = f2_sub(p1, p2);
    im = f2_sub(f2_neg(p3), p4);  // (-a.re) b.im = -(a.re b.im) exactly
  }
  if (minus) {
    xre = f2_sub(xre, re);
    xim = f2_sub(xim, im);
  } else {
    xre = f2_add(xre, re);
    xim = f2_add(xim, im);
  }
}
// the same on float2 values (one complex a)
template <bool CA, bool CB>
__device__ __forceinline__ void cmac_x2(float2& xre, float2& xim, bool minus, Cx<float> a, float2 bre, float2 bim,
                                        float z) {
  F2 r = f2_pack(xre.x, xre.y), i = f2_pack(xim.x, xim.y);
  cmac_f2<CA, CB>(r, i, minus, f2_pack(a.re, a.re), f2_pack(a.im, a.im), f2_pack(bre.x, bre.y),
                  f2_pack(bim.x, bim.y), f2_pack(z, z));
  xre = make_float2(f2_lo(r), f2_hi(r));
  xim = make_float2(f2_lo(i), f2_hi(i));
}

// one complex number as a single 8-B (F3) / 16-B (D3) access (the address
// is aligned to the complex number's size)
template <typename R>
__device__ __forceinline__ Cx<R> ldc(const Cx<R>* q) {
  if constexpr (sizeof(R) == 4) {
    const float2 v = *reinterpret_cast<const float2*>(q);
    return Cx<R>{v.x, v.y};
  } else {
    const double2 v = *reinterpret_cast<const double2*>(q);
    return Cx<R>{v.x, v.y};
  }
}
// two consecutive complex numbers (16-B aligned): one 16-B access in F3
template <typename R>
__device__ __forceinline__ void ldc2(const Cx<R>* q, Cx<R>& u, Cx<R>& v) {
  if constexpr (sizeof(R) == 4) {
    const float4 w = *reinterpret_cast<const float4*>(q);
    u = Cx<R>{w.x, w.y};
    v = Cx<R>{w.z, w.w};
  } else {
    const double2 a = reinterpret_cast<const double2*>(q)[0], b = reinterpret_cast<const double2*>(q)[1];
    u = Cx<R>{a.x, a.y};
    v = Cx<R>{b.x, b.y};
  }
}
template <typename R>
__device__ __forceinline__ void stc2(Cx<R>* q, Cx<R> u, Cx<R> v) {
  if constexpr (sizeof(R) == 4) {
    *reinterpret_cast<float4*>(q) = make_float4(u.re, u.im, v.re, v.im);
  } else {
    reinterpret_cast<double2*>(q)[0] = make_double2(u.re, u.im);
    reinterpret_cast<double2*>(q)[1] = make_double2(v.re, v.im);
  }
}
template <typename R>
__device__ __forceinline__ void stc(Cx<R>* q, Cx<R> v) {
  if constexpr (sizeof(R) == 4)
    *reinterpret_cast<float2*>(q) = make_float2(v.re, v.im);
  else
    *reinterpret_cast<double2*>(q) = make_double2(v.re, v.im);
}

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

// two consecutive complex numbers e, e+1 of record k (16 B F3, 32 B D3)
template <typename R>
__device__ __forceinline__ void ld2(Cx<R> (&v)[2], const Opnd& o, long long k, int e, int rec, bool vec) {
  if (vec) {
    const Cx<R>* base = static_cast<const Cx<R>*>(o.base) + k * rec + e;
    if constexpr (sizeof(R) == 4) {
      const float4 u = __ldg(reinterpret_cast<const float4*>(base));
      v[0] = Cx<R>{u.x, u.y};
      v[1] = Cx<R>{u.z, u.w};
    } else {
      const double2* q = reinterpret_cast<const double2*>(base);
      const double2 u = __ldg(q), w = __ldg(q + 1);
      v[0] = Cx<R>{u.x, u.y};
      v[1] = Cx<R>{w.x, w.y};
    }
  } else {
    v[0] = ld_elem<R>(o, k, e, rec);
    v[1] = ld_elem<R>(o, k, e + 1, rec);
  }
}
template <typename R>
__device__ __forceinline__ void ld2_out(Cx<R> (&v)[2], const Cx<R>* q, bool vec) {
  if (vec) {
    if constexpr (sizeof(R) == 4) {
      const float4 u = *reinterpret_cast<const float4*>(q);
      v[0] = Cx<R>{u.x, u.y};
      v[1] = Cx<R>{u.z, u.w};
    } else {
      const double2 u = reinterpret_cast<const double2*>(q)[0], w = reinterpret_cast<const double2*>(q)[1];
      v[0] = Cx<R>{u.x, u.y};
      v[1] = Cx<R>{w.x, w.y};
    }
  } else {
    v[0] = q[0];
    v[1] = q[1];
  }
}
template <typename R>
__device__ __forceinline__ void st2(Cx<R>* q, const Cx<R> (&v)[2], bool vec) {
  if (vec) {
    if constexpr (sizeof(R) == 4) {
      *reinterpret_cast<float4*>(q) = make_float4(v[0].re, v[0].im, v[1].re, v[1].im);
    } else {
      reinterpret_cast<double2*>(q)[0] = make_double2(v[0].re, v[0].im);
      reinterpret_cast<double2*>(q)[1] = make_double2(v[1].re, v[1].im);
    }
  } else {
    q[0] = v[0];
    q[1] = v[1];
  }
}

template <typename R>
__device__ __forceinline__ void init2(Cx<R> (&x)[2], const Cx<R>* q, bool load, bool vec) {
  if (load) {
    ld2_out<R>(x, q, vec);
  } else {
    x[0] = Cx<R>{R(0), R(0)};
    x[1] = Cx<R>{R(0), R(0)};
  }
}

// M * P: 24 threads per site; thread q = (is, jc, jh), outputs (ic, is, jc,
// 2jh..2jh+1) for ic = 0..2
template <typename R, bool CA, bool CB>
__global__ void __launch_bounds__(256) prop_mp_kernel(const PropParams p) {
  const long long total = p.n * 24;
  const bool minus = (p.eqop == MEQ || p.eqop == EQM);
  const bool load = (p.eqop == PEQ || p.eqop == MEQ);
  const long long stride = (long long)gridDim.x * blockDim.x;
  // two elements per iteration (g and g + stride): both elements' operand
  // loads are issued before either's arithmetic, twice the bytes in flight
  for (long long g0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; g0 < total; g0 += 2 * stride) {
    constexpr int U = 2;
    long long kk[U];
    int qq[U];
    bool on[U];
    Cx<R> mm[U][9], bb[U][3][2];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const long long g = g0 + u * stride;
      on[u] = g < total;
      const long long i = on[u] ? g / 24 : 0;
      qq[u] = (int)(g - i * 24);
      kk[u] = !on[u] ? 0 : p.gang ? (long long)p.gang[i] : i;
      if (!on[u]) continue;
      const int q = qq[u], is = q / 6, jc = (q >> 1) % 3, jh = q & 1;
#pragma unroll
      for (int e = 0; e < 9; e++) mm[u][e] = ld_elem<R>(p.a, kk[u], e, 9);
#pragma unroll
      for (int kc = 0; kc < 3; kc++) {
        if constexpr (!CB) {
          ld2<R>(bb[u][kc], p.b, kk[u], kc * 48 + 2 * q, 144, p.vec_b);
        } else {
#pragma unroll
          for (int j = 0; j < 2; j++)
            bb[u][kc][j] = ld_elem<R>(p.b, kk[u], p_idx(kc, is, jc, 2 * jh + j, true), 144);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (!on[u]) continue;
      Cx<R>* out = static_cast<Cx<R>*>(p.out) + kk[u] * 144 + 2 * qq[u];  // + ic * 48
      Cx<R> x[3][2];
#pragma unroll
      for (int ic = 0; ic < 3; ic++) init2<R>(x[ic], out + ic * 48, load, p.vec_out);
#pragma unroll
      for (int kc = 0; kc < 3; kc++)
#pragma unroll
        for (int ic = 0; ic < 3; ic++)
#pragma unroll
          for (int j = 0; j < 2; j++) cmac<CA, CB>(x[ic][j], minus, mm[u][m_idx(ic, kc, CA)], bb[u][kc][j]);
#pragma unroll
      for (int ic = 0; ic < 3; ic++) st2<R>(out + ic * 48, x[ic], p.vec_out);
    }
  }
}

// P * M: 24 threads per site; thread q = (ic, is, jh), outputs (ic, is, jc,
// 2jh..2jh+1) for jc = 0..2
template <typename R, bool CA, bool CB>
__global__ void __launch_bounds__(256) prop_pm_kernel(const PropParams p) {
  const long long total = p.n * 24;
  const bool minus = (p.eqop == MEQ || p.eqop == EQM);
  const bool load = (p.eqop == PEQ || p.eqop == MEQ);
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const long long i = g / 24;
    const int q = (int)(g - i * 24);
    const int row = q >> 1, jh = q & 1;  // row = ic * 4 + is
    const int ic = row >> 2, is = row & 3;
    const long long k = p.gang ? (long long)p.gang[i] : i;
    Cx<R>* out = static_cast<Cx<R>*>(p.out) + k * 144 + row * 12 + 2 * jh;  // + jc * 4
    Cx<R> mm[9];
#pragma unroll
    for (int e = 0; e < 9; e++) mm[e] = ld_elem<R>(p.b, k, e, 9);
    Cx<R> x[3][2];
#pragma unroll
    for (int jc = 0; jc < 3; jc++) init2<R>(x[jc], out + jc * 4, load, p.vec_out);
#pragma unroll
    for (int kc = 0; kc < 3; kc++) {
      Cx<R> a[2];
      if constexpr (!CA) {
        ld2<R>(a, p.a, k, row * 12 + kc * 4 + 2 * jh, 144, p.vec_a);
      } else {
#pragma unroll
        for (int j = 0; j < 2; j++) a[j] = ld_elem<R>(p.a, k, p_idx(ic, is, kc, 2 * jh + j, true), 144);
      }
#pragma unroll
      for (int jc = 0; jc < 3; jc++)
#pragma unroll
        for (int j = 0; j < 2; j++) cmac<CA, CB>(x[jc][j], minus, a[j], mm[m_idx(kc, jc, CB)]);
    }
#pragma unroll
    for (int jc = 0; jc < 3; jc++) st2<R>(out + jc * 4, x[jc], p.vec_out);
  }
}

// P * P: thread (jc, js block) keeps the second operand's 12 runs
// B[kc][ks][jc][js block] in registers and streams the rows of the first
// operand, producing outputs (row, jc, js block) for all 12 rows.  The js
// block is two spin components in F3 (6 threads per site, 16-B runs) and one
// in D3 (12 threads per site, 16-B elements), which keeps the FP64 version's
// registers low enough for two blocks per SM.
template <typename R, bool CA, bool CB>
__global__ void __launch_bounds__(256) prop_pp_kernel(const PropParams p) {
  constexpr int JW = sizeof(R) == 4 ? 2 : 1;  // spin components per thread
  constexpr int TPS = 12 / JW;                 // threads per site
  const long long total = p.n * TPS;
  const bool minus = (p.eqop == MEQ || p.eqop == EQM);
  const bool load = (p.eqop == PEQ || p.eqop == MEQ);
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const long long i = g / TPS;
    const int q = (int)(g - i * TPS);
    const int jc = q / (4 / JW), js0 = (q % (4 / JW)) * JW;
    const long long k = p.gang ? (long long)p.gang[i] : i;
    Cx<R>* out = static_cast<Cx<R>*>(p.out) + k * 144 + jc * 4 + js0;  // + row * 12
    Cx<R> b[12][JW];
#pragma unroll
    for (int kk = 0; kk < 12; kk++) {  // kk = kc * 4 + ks
      if constexpr (!CB && JW == 2) {
        ld2<R>(b[kk], p.b, k, kk * 12 + jc * 4 + js0, 144, p.vec_b);
      } else {
#pragma unroll
        for (int j = 0; j < JW; j++) b[kk][j] = ld_elem<R>(p.b, k, p_idx(kk >> 2, kk & 3, jc, js0 + j, CB), 144);
      }
    }
    // rows of the first operand, the next row's loads issued before the
    // current row's multiply-adds so that a DRAM round trip overlaps them
    Cx<R> a[12], an[12];
    auto load_row = [&](Cx<R>(&dst)[12], int row) {
#pragma unroll
      for (int kk = 0; kk < 12; kk += 2) {
        if constexpr (!CA) {
          Cx<R> t[2];
          ld2<R>(t, p.a, k, row * 12 + kk, 144, p.vec_a);
          dst[kk] = t[0];
          dst[kk + 1] = t[1];
        } else {
#pragma unroll
          for (int j = 0; j < 2; j++)
            dst[kk + j] = ld_elem<R>(p.a, k, p_idx(row >> 2, row & 3, (kk + j) >> 2, (kk + j) & 3, true), 144);
        }
      }
    };
    load_row(a, 0);
    if constexpr (sizeof(R) == 4) {
      // F3: both output columns in packed FP32x2 arithmetic (cmac_x2)
      float2 bre[12], bim[12];
#pragma unroll
      for (int kk = 0; kk < 12; kk++) {
        bre[kk] = make_float2(b[kk][0].re, b[kk][1].re);
        bim[kk] = make_float2(b[kk][0].im, b[kk][1].im);
      }
#pragma unroll 1
      for (int row = 0; row < 12; row++) {
        if (row + 1 < 12) load_row(an, row + 1);
        float2 xre = make_float2(0.f, 0.f), xim = make_float2(0.f, 0.f);
        if (load) {
          Cx<R> x0[2];
          ld2_out<R>(x0, out + row * 12, p.vec_out);
          xre = make_float2(x0[0].re, x0[1].re);
          xim = make_float2(x0[0].im, x0[1].im);
        }
#pragma unroll
        for (int kk = 0; kk < 12; kk++) cmac_x2<CA, CB>(xre, xim, minus, a[kk], bre[kk], bim[kk], p.negzero);
        const Cx<R> x[2] = {Cx<R>{xre.x, xim.x}, Cx<R>{xre.y, xim.y}};
        st2<R>(out + row * 12, x, p.vec_out);
#pragma unroll
        for (int kk = 0; kk < 12; kk++) a[kk] = an[kk];
      }
      continue;
    }
#pragma unroll 1
    for (int row = 0; row < 12; row++) {
      if (row + 1 < 12) load_row(an, row + 1);
      Cx<R> x[JW];
      if (load) {
#pragma unroll
        for (int j = 0; j < JW; j++) x[j] = out[row * 12 + j];
      } else {
#pragma unroll
        for (int j = 0; j < JW; j++) x[j] = Cx<R>{R(0), R(0)};
      }
#pragma unroll
      for (int kk = 0; kk < 12; kk++)
#pragma unroll
        for (int j = 0; j < JW; j++) cmac<CA, CB>(x[j], minus, a[kk], b[kk][j]);
      if constexpr (JW == 2) {
        st2<R>(out + row * 12, x, p.vec_out);
      } else {
        out[row * 12] = x[0];
      }
#pragma unroll
      for (int kk = 0; kk < 12; kk++) a[kk] = an[kk];
    }
  }
}

// Propagator products (P * P, M * P, P * M; F3 and D3) for contiguous, 16-B
// aligned operands without a gang index: bulk-copy (TMA) pipeline,
// persistent, warp-specialised like the site engine.
// Block = 12 * SPB consumer threads (12 per site of a tile of SPB sites) + one
// producer warp.  Per stage of the ring there is a `full` mbarrier (completed
// by the copies' transaction bytes) and an `empty` mbarrier (one arrival per
// consumer warp).  The producer issues one bulk copy per P record and one per
// tile for the M records into the stage (slots padded so that the sites one
// warp covers spread over the banks, PTSlots); consumers wait on `full`,
// compute from the stage, release it and store their results with 16-B
// stores.  No block barrier sits in the tile loop.  F3 P * P: the producer
// then rewrites each landed second-operand record in place into
// per-column-pair real / imaginary planes and arrives on a third mbarrier,
// `ready`, which the consumers wait on instead of `full`.
//
// P * P: in F3 thread (rg, cg) of a site (12 per site) accumulates the 12
// output elements of rows 2rg, 2rg+1 at the column pairs {2(cg + 2q),
// 2(cg + 2q) + 1}, q = 0..2, two columns per FP32x2 register (cmac_f2:
// per-lane rounding as cmac<CA, CB>); in D3 thread (r, cg) (24 per site)
// accumulates row r at the columns cg + 2q, q = 0..5, with cmac<CA, CB>.  M * P and
// P * M: see the consumer branch.  Every element is accumulated over k in
// order as the reference does, so results are bit-identical.  Every wait is
// time-bounded; a failed wait raises the block's abort flag, which ends every
// other wait of the block at once, and loads still in flight are drained
// (bounded) before the block exits.
//
// Dynamic shared memory: [full[8] | empty[8] | abort flag | ready[8] at
//                         192 B | pad to 256 B | stages x (SPB x (SA + SB)
//                         bytes)].
// Stage slots of the bulk-copy kernel per operand: record bytes and slot
// stride (bytes), chosen so that the sites one warp covers spread over the
// shared-memory banks.  P records, one bulk copy per site into padded slots:
// F3 1168 (first operand of P * P, M * P and P * M) / 1184 (second operand of
// P * P), D3 2336.  M records (72 / 144 B, not a multiple of 16), one bulk
// copy per full tile into consecutive slots: three sites 72 / 144 B apart
// read distinct banks.
template <typename R, int KIND>
struct PTSlots {
  static constexpr unsigned PREC = 144 * sizeof(Cx<R>), MREC = 9 * sizeof(Cx<R>);
  static constexpr unsigned PSLOT_A = sizeof(R) == 4 ? 1168 : 2336, PSLOT_B = sizeof(R) == 4 ? 1184 : 2336;
  static constexpr unsigned MSLOT = MREC;
  static constexpr unsigned RA = KIND == PK_MP ? MREC : PREC;  // first operand
  static constexpr unsigned RB = KIND == PK_PM ? MREC : PREC;  // second operand
  static constexpr unsigned A = KIND == PK_MP ? MSLOT : PSLOT_A;
  static constexpr unsigned B = KIND == PK_PM ? MSLOT : (KIND == PK_PP ? PSLOT_B : PSLOT_A);
};

// consumer threads per site: 24 for D3 P * P (one output row each: twice the
// warps in the same shared memory for its FP64 dependency chains) and for
// M * P and P * M (a thread's outputs are two consecutive elements of three
// rows, so that adjacent lanes write adjacent 16-B / 32-B runs), else 12
template <typename R, int KIND>
constexpr int prop_tma_tps() {
  // (F3 P * P at 24 threads per site, one row each, measured slower: 98 us
  // against 87 us at 12)
  return (KIND == PK_MP || KIND == PK_PM || sizeof(R) == 8) ? 24 : 12;
}

template <typename R, int KIND, bool CA, bool CB, int SPB, int MINB>
__global__ void __launch_bounds__(prop_tma_tps<R, KIND>() * SPB + 32, MINB)
    prop_tma_kernel(const PropParams p, long long ntiles) {
  extern __shared__ __align__(128) unsigned char ptm[];
  constexpr int TPS = prop_tma_tps<R, KIND>();
  constexpr int NCT = TPS * SPB;  // consumer threads
  constexpr int NCW = NCT / 32;  // consumer warps
  using SL = PTSlots<R, KIND>;
  constexpr unsigned RA = SL::RA, RB = SL::RB;  // bytes per record of each operand
  constexpr unsigned SA = SL::A, SB = SL::B;
  constexpr unsigned STAGE = SPB * (SA + SB);
  // per-site (P) slots start on 16 B; the M slots of a tile form one region
  // whose size keeps the next region on 16 B
  static_assert((KIND == PK_MP ? (SPB * SA) % 16 : SA % 16) == 0 &&
                    (KIND == PK_PM ? (SPB * SB) % 16 : SB % 16) == 0 && SA >= RA && SB >= RB,
                "stage slots keep 16-B alignment");
  static_assert(NCT % 32 == 0, "consumer threads fill whole warps");
  static_assert(2 * SPB <= 32, "one producer lane per site and operand");
  const int S = p.stages;
  uint64_t* full = reinterpret_cast<uint64_t*>(ptm);
  uint64_t* empty = full + 8;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(ptm + 8 * 16);
  uint64_t* ready = reinterpret_cast<uint64_t*>(ptm + 8 * 24);  // F3 P * P: second operand rewritten
  unsigned char* stages = ptm + 256;
  // F3 P * P: the producer warp rewrites each landed second-operand record
  // in place into per-column-pair real / imaginary planes, so that the
  // consumers load ready FP32x2 operand pairs; consumers wait on `ready`
  constexpr bool XF = KIND == PK_PP && sizeof(R) == 4;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long my = ((long long)blockIdx.x < ntiles) ? (ntiles - 1 - (long long)blockIdx.x) / gridDim.x + 1 : 0;
  if (tid == 0) {
    for (int i = 0; i < S; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], (unsigned)NCW);
      mbar_init(&ready[i], 1);
    }
    *abort_flag = 0;
    mbar_init_fence();
  }
  __syncthreads();
  long long issued = 0;
  if (warp == NCW) {
    // ------------------------------------------------------------ producer
    const uint64_t pol = policy_evict_first();
    const char* Ag = static_cast<const char*>(p.a.base);
    const char* Bg = static_cast<const char*>(p.b.base);
    // F3 P * P: once tile kt's copies have landed, rewrite its second-operand
    // records in place.  Element (kk, j) (of P, or of P^+ read transposed)
    // goes to floats kk*24 + cg*12 + 2q + (j & 1) (real) and 6 later
    // (imaginary), with j / 2 = cg + 2q: per k and column half cg, the real
    // parts of the three column pairs, then their imaginary parts.
    auto transform = [&](long long kt) -> bool {
      const int sst = (int)(kt % S);
      const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded_idle(&full[sst], (uint32_t)((kt / S) & 1), p.err,
                                                                      2000000000ull, abort_flag));
      if (!ok) return false;
      const long long s0 = ((long long)blockIdx.x + kt * gridDim.x) * SPB;
      const int nl = (int)((p.n - s0) < SPB ? (p.n - s0) : SPB);
      float* sbase = reinterpret_cast<float*>(stages + (size_t)sst * STAGE + SPB * SA);
      for (int site = 0; site < nl; site++) {
        float* b = sbase + site * (SB / 4);
        float4 v[3];
#pragma unroll
        for (int i = 0; i < 3; i++) {
          const int w = lane + 32 * i;  // 16-B word of the record: elements (r, c), (r, c + 1), c even
          if (w < 72) v[i] = reinterpret_cast<const float4*>(b)[w];
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 3; i++) {
          const int w = lane + 32 * i;
          if (w < 72) {
            const int r = w / 6, c = 2 * (w - r * 6);
            if constexpr (!CB) {  // (kk, j) = (r, c), (r, c + 1): one pair of each plane
              const int jp = c >> 1, o = r * 24 + (jp & 1) * 12 + 2 * (jp >> 1);
              *reinterpret_cast<float2*>(b + o) = make_float2(v[i].x, v[i].z);
              *reinterpret_cast<float2*>(b + o + 6) = make_float2(v[i].y, v[i].w);
            } else {  // P^+: (kk, j) = (c, r), (c + 1, r)
              const int jp = r >> 1, o = c * 24 + (jp & 1) * 12 + 2 * (jp >> 1) + (r & 1);
              b[o] = v[i].x;
              b[o + 6] = v[i].y;
              b[o + 24] = v[i].z;
              b[o + 30] = v[i].w;
            }
          }
        }
        __syncwarp();
      }
      // the rewritten slots: visible to the consumers through `ready`, and
      // ordered before the async proxy's next copy into the stage
      __threadfence_block();
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&ready[sst]);
      return true;
    };
    int st = 0;
    long long round = 0, k = 0;
    for (; k < my; k++) {
      bool ok = true;
      if (lane == 0 && round > 0)
        ok = mbar_wait_bounded_idle(&empty[st], (uint32_t)((round - 1) & 1), p.err, 2000000000ull, abort_flag);
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) {
        if (lane == 0) *abort_flag = 1;
        break;
      }
      const long long site0 = ((long long)blockIdx.x + k * gridDim.x) * SPB;
      const int nloc = (int)((p.n - site0) < SPB ? (p.n - site0) : SPB);
      unsigned char* sa = stages + (size_t)st * STAGE;
      unsigned char* sb = sa + SPB * SA;
      if (lane == 0) mbar_arrive_expect_tx(&full[st], (uint32_t)nloc * (RA + RB));
      __syncwarp();
      if constexpr (KIND == PK_PP) {
        if (lane < nloc)
          bulk_g2s(sa + lane * SA, Ag + (site0 + lane) * RA, RA, &full[st], pol);
        else if (lane >= SPB && lane - SPB < nloc)
          bulk_g2s(sb + (lane - SPB) * SB, Bg + (site0 + lane - SPB) * RB, RB, &full[st], pol);
      } else {
        // P records one per site; the M records of the tile (always a full
        // tile here: SPB x 72 / 144 B from a 16-B aligned start) in one copy
        constexpr bool MP = KIND == PK_MP;
        constexpr unsigned PREC = SL::PREC, MREC = SL::MREC, PS = MP ? SB : SA;
        unsigned char* pslots = MP ? sb : sa;
        unsigned char* mslots = MP ? sa : sb;
        const char* Pg = MP ? Bg : Ag;
        const char* Mg = MP ? Ag : Bg;
        if (lane < nloc)
          bulk_g2s(pslots + lane * PS, Pg + (site0 + lane) * PREC, PREC, &full[st], pol);
        else if (lane == 31)
          bulk_g2s(mslots, Mg + site0 * MREC, (unsigned)nloc * MREC, &full[st], pol);
      }
      if constexpr (XF) {
        if (k >= 1 && !transform(k - 1)) {  // the previous tile, while this one's copies fly
          if (lane == 0) *abort_flag = 1;
          k++;  // tile k's copies were issued
          break;
        }
      }
      if (++st == S) {
        st = 0;
        round++;
      }
    }
    issued = k;
    if constexpr (XF) {
      if (issued == my && my >= 1 && !transform(my - 1) && lane == 0) *abort_flag = 1;
    }
  } else {
    // ------------------------------------------------------------ consumers
    const int ls = tid / TPS, t12 = tid - ls * TPS, rg = t12 >> 1, cg = t12 & 1;  // (t12: 0 .. TPS-1)
    const bool minus = (p.eqop == MEQ || p.eqop == EQM);
    const bool load = (p.eqop == PEQ || p.eqop == MEQ);
    const F2 z2 = f2_pack(p.negzero, p.negzero);  // (F3 products)
    int st = 0;
    uint32_t par = 0;
    for (long long k = 0; k < my; k++) {
      // warp-uniform, so that the warp leaves the loop as a whole
      const bool ok = __all_sync(
          0xffffffffu, mbar_wait_bounded_idle(XF ? &ready[st] : &full[st], par, p.err, 2000000000ull, abort_flag));
      const long long site0 = ((long long)blockIdx.x + k * gridDim.x) * SPB;
      const int nloc = (int)((p.n - site0) < SPB ? (p.n - site0) : SPB);
      const bool active = ok && ls < nloc;
      const unsigned char* stg = stages + (size_t)st * STAGE;
      if constexpr (KIND == PK_PP && sizeof(R) == 4) {
        // rows RPT * rg + i of this thread (RPT = 1 with 24 threads per site)
        constexpr int RPT = TPS == 24 ? 1 : 2;
        const float* A = reinterpret_cast<const float*>(stg + ls * SA);
        const float* B = reinterpret_cast<const float*>(stg + SPB * SA + ls * SB);
        const Cx<float>* og = static_cast<const Cx<float>*>(p.out) + (site0 + ls) * 144 + 2 * cg;
        F2 xr[RPT][3], xi[RPT][3];  // [row RPT * rg + i][q]: lanes = columns 2(cg + 2q), +1
#pragma unroll
        for (int i = 0; i < RPT; i++)
#pragma unroll
          for (int q = 0; q < 3; q++) {
            if (load && active) {
              const float4 v = *reinterpret_cast<const float4*>(og + (RPT * rg + i) * 12 + 4 * q);
              xr[i][q] = f2_pack(v.x, v.z);
              xi[i][q] = f2_pack(v.y, v.w);
            } else {
              xr[i][q] = 0ull;  // (+0, +0)
              xi[i][q] = 0ull;
            }
          }
        if (active) {
#pragma unroll
          for (int kk = 0; kk < 12; kk += 2) {
            // element (row RPT * rg + i, kk + h) before conjugation, broadcast to both lanes
            F2 ar[RPT][2], ai[RPT][2];
            if constexpr (!CA) {
#pragma unroll
              for (int i = 0; i < RPT; i++) {
                const float4 v = *reinterpret_cast<const float4*>(A + ((RPT * rg + i) * 12 + kk) * 2);
                ar[i][0] = f2_pack(v.x, v.x);
                ai[i][0] = f2_pack(v.y, v.y);
                ar[i][1] = f2_pack(v.z, v.z);
                ai[i][1] = f2_pack(v.w, v.w);
              }
            } else if constexpr (RPT == 2) {
              // P^+[r][kk] = conj P[kk][r]: elements (kk + h, 2rg), (kk + h, 2rg + 1) are adjacent
#pragma unroll
              for (int h = 0; h < 2; h++) {
                const float4 v = *reinterpret_cast<const float4*>(A + ((kk + h) * 12 + 2 * rg) * 2);
                ar[0][h] = f2_pack(v.x, v.x);
                ai[0][h] = f2_pack(v.y, v.y);
                ar[1][h] = f2_pack(v.z, v.z);
                ai[1][h] = f2_pack(v.w, v.w);
              }
            } else {  // P^+[r][kk] = conj P[kk][r], one row
#pragma unroll
              for (int h = 0; h < 2; h++) {
                const float2 v = *reinterpret_cast<const float2*>(A + ((kk + h) * 12 + rg) * 2);
                ar[0][h] = f2_pack(v.x, v.x);
                ai[0][h] = f2_pack(v.y, v.y);
              }
            }
            // second-operand elements (kk + h, j), j = 2(cg + 2q) + {0, 1}, before
            // conjugation, from the planes the producer wrote: per (k, cg) the
            // real pairs of q = 0, 1, 2 then the imaginary pairs
            F2 bre[2][3], bim[2][3];
#pragma unroll
            for (int h = 0; h < 2; h++) {
              const ulonglong2* q2 = reinterpret_cast<const ulonglong2*>(B + (kk + h) * 24 + cg * 12);
              const ulonglong2 w0 = q2[0], w1 = q2[1], w2 = q2[2];
              bre[h][0] = w0.x;
              bre[h][1] = w0.y;
              bre[h][2] = w1.x;
              bim[h][0] = w1.y;
              bim[h][1] = w2.x;
              bim[h][2] = w2.y;
            }
#pragma unroll
            for (int h = 0; h < 2; h++)
#pragma unroll
              for (int i = 0; i < RPT; i++)
#pragma unroll
                for (int q = 0; q < 3; q++)
                  cmac_f2<CA, CB>(xr[i][q], xi[i][q], minus, ar[i][h], ai[i][h], bre[h][q], bim[h][q], z2);
          }
        }
        release_stage(&empty[st], lane);  // this warp is done with the stage
        if (!ok) {
          *abort_flag = 1;
          break;
        }
        if (ls < nloc) {
          Cx<float>* o = static_cast<Cx<float>*>(p.out) + (site0 + ls) * 144 + 2 * cg;
#pragma unroll
          for (int i = 0; i < RPT; i++)
#pragma unroll
            for (int q = 0; q < 3; q++)
              *reinterpret_cast<float4*>(o + (RPT * rg + i) * 12 + 4 * q) =
                  make_float4(f2_lo(xr[i][q]), f2_lo(xi[i][q]), f2_hi(xr[i][q]), f2_hi(xi[i][q]));
        }
      } else if constexpr (KIND == PK_PP) {
        // D3 (24 threads per site): thread (r, cg) = (rg, cg) accumulates row r
        // at columns cg + 2q, q = 0..5, with cmac<CA, CB>
        const int r = rg;
        const Cx<double>* A = reinterpret_cast<const Cx<double>*>(stg + ls * SA);
        const Cx<double>* B = reinterpret_cast<const Cx<double>*>(stg + SPB * SA + ls * SB);
        Cx<double>* o = static_cast<Cx<double>*>(p.out) + (site0 + ls) * 144 + r * 12 + cg;
        Cx<double> x[6];
#pragma unroll
        for (int q = 0; q < 6; q++) x[q] = (load && active) ? ldc(o + 2 * q) : Cx<double>{0.0, 0.0};
        if (active) {
#pragma unroll 4
          for (int kk = 0; kk < 12; kk++) {
            // element (r, kk) before conjugation (P^+[r][kk] = conj P[kk][r])
            const Cx<double> a = ldc(A + (CA ? kk * 12 + r : r * 12 + kk));
#pragma unroll
            for (int q = 0; q < 6; q++) {
              const int j = cg + 2 * q;  // P^+[kk][j] = conj P[j][kk]
              cmac<CA, CB>(x[q], minus, a, ldc(B + (CB ? j * 12 + kk : kk * 12 + j)));
            }
          }
        }
        release_stage(&empty[st], lane);  // this warp is done with the stage
        if (!ok) {
          *abort_flag = 1;
          break;
        }
        if (ls < nloc) {
#pragma unroll
          for (int q = 0; q < 6; q++) stc(o + 2 * q, x[q]);
        }
      } else {
        static_assert(KIND != PK_PP && TPS == 24, "M * P and P * M run 24 threads per site");
        // 24 threads per site, scalar cmac<CA, CB>, k in order.  M * P:
        // thread (is, jc, jh) accumulates outputs (ic, is, jc, 2jh + j),
        // ic = 0..2, from P'[kc][is][jc][2jh + j] and M'[ic][kc]; P * M: thread
        // (ic, is, jh) accumulates outputs (ic, is, jc, 2jh + j), jc = 0..2,
        // from P'[ic][is][kc][2jh + j] and M'[kc][jc] (P^+ read transposed)
        constexpr bool MP = KIND == PK_MP;
        const int g = t12 >> 1, jh = t12 & 1;  // g = is * 3 + jc (M * P) or ic * 4 + is (P * M)
        const int u = MP ? g / 3 : g >> 2, v = MP ? g - (g / 3) * 3 : g & 3;
        const Cx<R>* A = reinterpret_cast<const Cx<R>*>(stg + ls * SA);
        const Cx<R>* B = reinterpret_cast<const Cx<R>*>(stg + SPB * SA + ls * SB);
        const Cx<R>* P = MP ? B : A;
        Cx<R>* o = static_cast<Cx<R>*>(p.out) + (site0 + ls) * 144;
        // output w (ic for M * P, jc for P * M), elements 2jh, 2jh + 1
        auto oidx = [&](int w) { return (MP ? p_idx(w, u, v, 0, false) : p_idx(u, v, w, 0, false)) + 2 * jh; };
        Cx<R> x[3][2];
#pragma unroll
        for (int w = 0; w < 3; w++) {
          if (load && active) {
            ldc2(o + oidx(w), x[w][0], x[w][1]);
          } else {
            x[w][0] = Cx<R>{R(0), R(0)};
            x[w][1] = Cx<R>{R(0), R(0)};
          }
        }
        if (active) {
#pragma unroll
          for (int kc = 0; kc < 3; kc++) {
            Cx<R> pv[2], mv[3];
            constexpr bool adj = MP ? CB : CA;
            if constexpr (!adj) {
              ldc2(P + (MP ? p_idx(kc, u, v, 2 * jh, false) : p_idx(u, v, kc, 2 * jh, false)), pv[0], pv[1]);
            } else {
#pragma unroll
              for (int j = 0; j < 2; j++)
                pv[j] = ldc(P + (MP ? p_idx(kc, u, v, 2 * jh + j, true) : p_idx(u, v, kc, 2 * jh + j, true)));
            }
#pragma unroll
            for (int w = 0; w < 3; w++) mv[w] = MP ? ldc(A + m_idx(w, kc, CA)) : ldc(B + m_idx(kc, w, CB));
#pragma unroll
            for (int w = 0; w < 3; w++)
#pragma unroll
              for (int j = 0; j < 2; j++) {
                if constexpr (MP)
                  cmac<CA, CB>(x[w][j], minus, mv[w], pv[j]);
                else
                  cmac<CA, CB>(x[w][j], minus, pv[j], mv[w]);
              }
          }
        }
        release_stage(&empty[st], lane);  // this warp is done with the stage
        if (!ok) {
          *abort_flag = 1;
          break;
        }
        if (ls < nloc) {
#pragma unroll
          for (int w = 0; w < 3; w++) stc2(o + oidx(w), x[w][0], x[w][1]);
        }
      }
      if (++st == S) {
        st = 0;
        par ^= 1u;
      }
    }
  }
  __syncthreads();
  if (*abort_flag && warp == NCW && lane == 0) {
    // a wait failed: before the block's shared memory is released, wait
    // (bounded) until every load still in flight has landed
    for (long long kk = (issued > S ? issued - S : 0); kk < issued; kk++)
      if (!mbar_wait_bounded(&full[kk % S], (uint32_t)((kk / S) & 1), p.err, 200000000ull, nullptr))
        raise_dev_error(p.err, QLA_DEVERR_BULK_TIMEOUT);
  }
}

// shared-memory bytes of prop_tma_kernel<R, KIND, .., SPB> with `stages` stages
template <typename R, int KIND>
constexpr size_t prop_tma_smem(int spb, int stages) {
  return 256 + (size_t)stages * spb * (PTSlots<R, KIND>::A + PTSlots<R, KIND>::B);
}

// blocks per SM of a kernel at (threads, smem), raising its dynamic
// shared-memory limit once per device
inline int prop_blocks_per_sm(const void* fn, int threads, size_t smem) {
  static std::mutex mu;
  static std::map<std::tuple<int, const void*, int, size_t>, int> cache;
  const int dev = current_device();
  std::lock_guard<std::mutex> g(mu);
  const auto key = std::make_tuple(dev, fn, threads, smem);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  if (smem > 48 * 1024) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, smem) != cudaSuccess || nb < 1) nb = 1;
  cudaGetLastError();
  cache[key] = nb;
  return nb;
}

// the spin trace: one thread per output element (9 per site)
template <typename R>
__global__ void __launch_bounds__(256) prop_trace_kernel(const PropParams p) {
  const long long total = p.n * 9;
  const bool minus = (p.eqop == MEQ || p.eqop == EQM);
  const bool load = (p.eqop == PEQ || p.eqop == MEQ);
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const long long i = g / 9;
    const int e = (int)(g - i * 9);
    const long long k = p.gang ? (long long)p.gang[i] : i;
    Cx<R>* out = static_cast<Cx<R>*>(p.out) + k * 9 + e;
    Cx<R> x = load ? *out : Cx<R>{R(0), R(0)};
    const int ic = e / 3, jc = e % 3;
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const Cx<R> v = ld_elem<R>(p.a, k, ((ic * 4 + s) * 3 + jc) * 4 + s, 144);
      if (minus) {
        x.re = rsub(x.re, v.re);
        x.im = rsub(x.im, v.im);
      } else {
        x.re = radd(x.re, v.re);
        x.im = radd(x.im, v.im);
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
  p.vec_out = (reinterpret_cast<uintptr_t>(r) & 15u) == 0;
  p.vec_a = a.mode == OM_CONTIG && (reinterpret_cast<uintptr_t>(a.base) & 15u) == 0;
  p.vec_b = b.mode == OM_CONTIG && (reinterpret_cast<uintptr_t>(b.base) & 15u) == 0;
  p.negzero = -0.0f;
  const int per_site = KIND == PK_TRACE ? 9 : KIND == PK_PP ? (sizeof(R) == 4 ? 6 : 12) : 24;
  const long long total = (long long)n * per_site;
  long long grid = (total + 255) / 256;
  const long long cap = (long long)device_sm_count() * 16;
  if (grid > cap) grid = cap;
  const unsigned gr = (unsigned)(grid < 1 ? 1 : grid);
  cudaStream_t st = current_stream();
  const bool contig =
      gang == nullptr && a.mode == OM_CONTIG && b.mode == OM_CONTIG && p.vec_a && p.vec_b && p.vec_out;
  if constexpr (KIND == PK_TRACE) {
    prop_trace_kernel<R><<<gr, 256, 0, st>>>(p);
  } else if (!contig) {
    // gang, pointer or unaligned operands: the direct kernels
    if constexpr (KIND == PK_MP)
      prop_mp_kernel<R, CA, CB><<<gr, 256, 0, st>>>(p);
    else if constexpr (KIND == PK_PM)
      prop_pm_kernel<R, CA, CB><<<gr, 256, 0, st>>>(p);
    else
      prop_pp_kernel<R, CA, CB><<<gr, 256, 0, st>>>(p);
  } else {
    // bulk-copy pipeline, tiles of 8 sites, 96 consumer threads + one
    // producer warp per block.  P * P: F3 three stages (57 KB), four blocks
    // per SM at up to 128 registers; measured on B200 (131,072 sites) 86 us
    // with the producer's rewrite of the second operand into planes, where
    // two stages took 109 us and four stages at three blocks per SM 99 us
    // (before the rewrite: 90 us; five or six blocks per SM at 80-96
    // registers 95-98 us); D3 two stages (75 KB), three blocks per SM.  M * P
    // and P * M (24 threads per site), where fewer requests in flight
    // measured faster (131,072 sites, M * P / P * M): F3 two stages and four
    // blocks per SM 52.5 / 52.6 us = 0.91 of HBM peak (three stages and three
    // blocks 53.3 / 53.4 us); D3 two stages and two blocks per SM 99.4 / 101.5
    // us = 0.96 / 0.94 (three stages and three blocks 107.4 / 114.8 us).
    constexpr int SPB = 8;
    constexpr bool F32 = sizeof(R) == 4;
    constexpr bool PP = KIND == PK_PP;
    constexpr int MINB = PP ? (F32 ? 4 : 3) : 3;
    constexpr int CAP = PP ? 32 : (F32 ? 4 : 2);  // blocks per SM at most
    p.stages = PP ? (F32 ? 3 : 2) : 2;
    p.err = device_error_word();
    const size_t smem = prop_tma_smem<R, KIND>(SPB, p.stages);
    // M * P and P * M: full tiles in the pipeline (the M records of a tile go
    // in one bulk copy), the last n % SPB sites by the direct kernel
    const long long ntiles = PP ? ((long long)n + SPB - 1) / SPB : (long long)n / SPB;
    if (ntiles > 0) {
      const void* fn = reinterpret_cast<const void*>(&prop_tma_kernel<R, KIND, CA, CB, SPB, MINB>);
      constexpr int NT = prop_tma_tps<R, KIND>() * SPB + 32;
      const int nb = prop_blocks_per_sm(fn, NT, smem);
      long long blocks = (long long)(nb < CAP ? nb : CAP) * device_sm_count();
      if (blocks > ntiles) blocks = ntiles;
      prop_tma_kernel<R, KIND, CA, CB, SPB, MINB><<<(unsigned)blocks, NT, smem, st>>>(p, ntiles);
    }
    if constexpr (!PP) {
      const long long done = ntiles * SPB;
      if (done < n) {
        using SL = PTSlots<R, KIND>;
        PropParams t = p;
        t.a.base = static_cast<const char*>(a.base) + done * SL::RA;
        t.b.base = static_cast<const char*>(b.base) + done * SL::RB;
        t.out = static_cast<Cx<R>*>(r) + done * 144;
        t.n = n - done;
        if constexpr (KIND == PK_MP)
          prop_mp_kernel<R, CA, CB><<<1, 256, 0, st>>>(t);
        else
          prop_pm_kernel<R, CA, CB><<<1, 256, 0, st>>>(t);
      }
    }
  }
  check_launch(kid);
}

}  // namespace qlab
