// qla_batch.cu -- many fields of uneven volume, each running its own short
// sequence of level-1 operations, in one persistent launch.
//
// A lattice code often applies a short level-1 sequence to many independent
// fields (sub-lattices, sources, time slices).  Launching QLA's functions
// once per field and step costs a launch each and leaves the GPU idle on the
// small fields.  Here a plan flattens every field's tiles into one global
// tile list (prefix sums over per-field tile counts) and one persistent,
// warp-specialised bulk-copy pipeline walks that list.  Each field carries a
// small program (qlagpu_F3_batch_program): streams (its record arrays, some
// gathered through an int32 index) and steps drawn from the engine's per-site
// operators -- colour-matrix left multiplication (lmult_site), spin
// projection and reconstruction (the SpprojOp / SpreconOp bodies), real
// multiples and copies -- so a field's results are bit-identical to the
// separate QLA_F3 calls the steps stand for.
//
// Per tile the producer lane copies, with 1-D bulk copies into the next
// pipeline stage, every contiguous input stream of the field, the index tile
// of every gathered stream and the old values of every INOUT stream.  The
// consumer warps run the program one site per lane: operands come from the
// stage, from gathers (read-only global loads at the staged index) or from
// two per-site registers; stored results go through a per-warp
// per-warp shared slice and one bulk store per output stream.  Steps
// only see values of the same site, so sites are independent and the launch
// needs no grid-wide ordering.  Partial tiles, and fields whose arrays are
// not 16-B aligned, run the same program with plain loads and stores.
//
// The launch (qlagpu_batch_run) passes only the plan's device table: it can
// be replayed from a captured CUDA graph.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <type_traits>
#include <vector>

#include "../../include/qla_b200_runtime.h"
#include "qla_launch.cuh"
#include "qla_ops.cuh"

namespace qlab {

constexpr int kMaxStreams = 8, kMaxSteps = 8, kMaxFields = 1024;
constexpr int kReg0 = 8, kReg1 = 9;
enum BKind : int { BK_V = 0, BK_H = 1, BK_D = 2, BK_M = 3 };
enum BRole : int { BR_IN = 0, BR_OUT = 1, BR_INOUT = 2 };
enum BOp : int { BOP_LMULT = 0, BOP_SPPROJ = 1, BOP_SPRECON = 2, BOP_RTIMES = 3, BOP_COPY = 4 };
// complex numbers per V, H, D, M record (F3)
__host__ __device__ constexpr int kncplx(int kind) { return kind == BK_V ? 3 : kind == BK_H ? 6 : kind == BK_D ? 12 : 9; }

struct BStream {
  char* base;
  const int* idx;
  long long nsrc;
  int kind, role;
  unsigned stage_off;  // contiguous IN / INOUT: record tile; gathered IN: index tile
  unsigned out_off;    // OUT / INOUT: this stream's part of a warp's output slice
};

struct BStep {
  int op, eqop, a, b, dst, store, adja, adjb, mu, sign;
  int kind_a, kind_b, kind_r;  // operand and result kinds (checked on the host)
  int load_stream;             // peq / meq: the old value comes from this INOUT stream's tile, else -1
  int spill;                   // a later step other than the next one reads this result's register
  int src_a, src_b;            // SrcKind of the operands (classified by the planner)
  float r;
};

struct alignas(16) BField {
  BStream s[kMaxStreams];
  BStep st[kMaxSteps];
  int nstreams, nsteps;
  long long n, tile0;
  unsigned tx_bytes;  // bytes the producer copies per full tile
  int direct;         // some base not 16-B aligned: every tile by plain loads
  int shape;          // ShapeId of this field's program (SH_GENERIC: none of the catalogue)
};

struct BatchParams {
  const BField* fields;
  int nfields;
  long long ntiles;
  int stages;
  unsigned stage_bytes, out_slice_bytes;  // out slice: 32 sites of every output stream
  int spill_regs;                         // some program keeps a register in shared memory
  long long chunk;                        // consecutive tiles per group dealt to a block
  unsigned* err;
};

struct BatchPlan {
  BField* dfields;
  int nfields;
  long long ntiles;
  int threads, stages, grid;
  unsigned stage_bytes, out_slice_bytes;
  int spill_regs;
  long long chunk;  // see BatchParams
  int mc;     // record capacity of the kernel instance: 9 or 12 complex numbers
  int shape;  // ShapeId of the kernel instance (SH_GENERIC: the interpreter)
  size_t smem;
};

// The field of tile g given the previous answer f (or -1): tiles come in
// runs, so a range check usually settles it without the search.
__device__ __forceinline__ int find_field(const long long* tile0, int nf, long long g);
__device__ __forceinline__ int field_of(const long long* tile0, int nf, long long g, int f) {
  if (f >= 0 && tile0[f] <= g && (f + 1 == nf || g < tile0[f + 1])) return f;
  return find_field(tile0, nf, g);
}
__device__ __forceinline__ int find_field(const long long* tile0, int nf, long long g) {
  int lo = 0, hi = nf - 1;  // last field with tile0 <= g
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tile0[mid] <= g)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// One record of any kind the plan uses, MC complex numbers long: 12 when
// some field uses DiracFermions, else 9 (colour matrices are the longest),
// which keeps the kernel's registers down for V / H / M programs.
template <int MC>
using Rec = Cx<float>[MC];


// --- record movement with a compile-time length N (complex numbers)
template <int N, int MC>
__device__ __forceinline__ void ld_smem(Rec<MC>& x, const unsigned char* p) {
  if constexpr (N % 2 == 0) {  // H, D: 16-B multiples
    const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
    for (int e = 0; e < N / 2; e++) {
      const float4 v = q[e];
      x[2 * e] = Cx<float>{v.x, v.y};
      x[2 * e + 1] = Cx<float>{v.z, v.w};
    }
  } else {
    const float2* q = reinterpret_cast<const float2*>(p);
#pragma unroll
    for (int e = 0; e < N; e++) {
      const float2 v = q[e];
      x[e] = Cx<float>{v.x, v.y};
    }
  }
}
template <int N, int MC>
__device__ __forceinline__ void st_smem(unsigned char* p, const Rec<MC>& y) {
  if constexpr (N % 2 == 0) {
    float4* q = reinterpret_cast<float4*>(p);
#pragma unroll
    for (int e = 0; e < N / 2; e++) q[e] = make_float4(y[2 * e].re, y[2 * e].im, y[2 * e + 1].re, y[2 * e + 1].im);
  } else {
    float2* q = reinterpret_cast<float2*>(p);
#pragma unroll
    for (int e = 0; e < N; e++) q[e] = make_float2(y[e].re, y[e].im);
  }
}
template <int N, int MC>
__device__ __forceinline__ void ld_global(Rec<MC>& x, const void* p) {
  const float2* q = reinterpret_cast<const float2*>(p);
#pragma unroll
  for (int e = 0; e < N; e++) {
    const float2 v = __ldg(q + e);
    x[e] = Cx<float>{v.x, v.y};
  }
}
template <int N, int MC>
__device__ __forceinline__ void ld_global_rw(Rec<MC>& x, const void* p) {  // a stream this launch also writes
  const float2* q = reinterpret_cast<const float2*>(p);
#pragma unroll
  for (int e = 0; e < N; e++) {
    const float2 v = q[e];
    x[e] = Cx<float>{v.x, v.y};
  }
}
template <int N, int MC>
__device__ __forceinline__ void st_global(void* p, const Rec<MC>& y) {
  float2* q = reinterpret_cast<float2*>(p);
#pragma unroll
  for (int e = 0; e < N; e++) q[e] = make_float2(y[e].re, y[e].im);
}
template <int MC>
__device__ __forceinline__ void zero_rec(Rec<MC>& x) {
#pragma unroll
  for (int e = 0; e < MC; e++) x[e] = Cx<float>{0.f, 0.f};
}
template <int MC>
__device__ __forceinline__ void copy_rec(Rec<MC>& x, const Rec<MC>& y) {
#pragma unroll
  for (int e = 0; e < MC; e++) x[e] = y[e];
}
template <int N, int MC>  // the first N complex numbers only
__device__ __forceinline__ void copy_rec_n(Rec<MC>& x, const Rec<MC>& y) {
#pragma unroll
  for (int e = 0; e < N; e++) x[e] = y[e];
}

// Where one site's operands live: the staged tile (stage != nullptr, lane
// t) or global memory (site i).  Step registers: the previous step's result
// stays in registers (`prev`); a result that a later, non-adjacent step reads
// is also kept in shared memory, element-major (element e of register k of
// thread t at regs + ((k * 12 + e) * T + t) * 8), so a warp touches
// consecutive words.
struct SiteSrc {
  const unsigned char* stage;
  int t;
  long long i;
  unsigned* err;
  unsigned char* regs;
  int T;
};
template <int N, int MC>
__device__ __forceinline__ void reg_load(Rec<MC>& x, const SiteSrc& src, int slot) {
  const float2* q = reinterpret_cast<const float2*>(src.regs) + (size_t)slot * 12 * src.T + src.t;
#pragma unroll
  for (int e = 0; e < N; e++) {
    const float2 v = q[(size_t)e * src.T];
    x[e] = Cx<float>{v.x, v.y};
  }
}
template <int N, int MC>
__device__ __forceinline__ void reg_store(const SiteSrc& src, int slot, const Rec<MC>& y) {
  float2* q = reinterpret_cast<float2*>(src.regs) + (size_t)slot * 12 * src.T + src.t;
#pragma unroll
  for (int e = 0; e < N; e++) q[(size_t)e * src.T] = make_float2(y[e].re, y[e].im);
}

// record of stream S at this site, as an input (gathered through its index)
template <int N, int MC>
__device__ __forceinline__ void fetch_stream(Rec<MC>& x, const BStream& S, const SiteSrc& src) {
  if (S.idx) {
    long long j = src.stage ? reinterpret_cast<const int*>(src.stage + S.stage_off)[src.t] : S.idx[src.i];
    if (S.nsrc > 0 && (j < 0 || j >= S.nsrc)) {
      raise_dev_error(src.err, QLA_DEVERR_BAD_INDEX);
      zero_rec(x);
      return;
    }
    ld_global<N>(x, S.base + j * (long long)(N * 8));
  } else if (src.stage) {
    ld_smem<N>(x, src.stage + S.stage_off + (unsigned)src.t * (N * 8));
  } else if (S.role == BR_INOUT) {
    ld_global_rw<N>(x, S.base + src.i * (N * 8));
  } else {
    ld_global<N>(x, S.base + src.i * (N * 8));
  }
}
// operand `ref` (a stream, or a register) of kind `kind`; prev / prev_reg:
// the previous step's result and its register
template <int N, int MC>
__device__ __forceinline__ void fetch_n(Rec<MC>& x, int ref, const BField& F, const SiteSrc& src,
                                        const Rec<MC>& prev, int prev_reg) {
  if (ref == prev_reg)
    copy_rec(x, prev);
  else if (ref >= kReg0)
    reg_load<N>(x, src, ref - kReg0);
  else
    fetch_stream<N>(x, F.s[ref], src);
}
template <int MC>
__device__ __forceinline__ void fetch(Rec<MC>& x, int ref, int kind, const BField& F, const SiteSrc& src,
                                      const Rec<MC>& prev, int prev_reg) {
  switch (kind) {
    case BK_V: fetch_n<3>(x, ref, F, src, prev, prev_reg); break;
    case BK_H: fetch_n<6>(x, ref, F, src, prev, prev_reg); break;
    case BK_M: fetch_n<9>(x, ref, F, src, prev, prev_reg); break;
    default:
      if constexpr (MC >= 12) fetch_n<12>(x, ref, F, src, prev, prev_reg);
      break;
  }
}
template <int MC>
__device__ __forceinline__ void set_reg(const SiteSrc& src, int slot, int kind, const Rec<MC>& y) {
  switch (kind) {
    case BK_V: reg_store<3>(src, slot, y); break;
    case BK_H: reg_store<6>(src, slot, y); break;
    case BK_M: reg_store<9>(src, slot, y); break;
    default:
      if constexpr (MC >= 12) reg_store<12>(src, slot, y);
      break;
  }
}

// --- the per-site arithmetic of each step kind (the engine's operators)
template <int N, int MC>
__device__ __forceinline__ void rtimes_n(int eqop, float at, const Rec<MC>& b, Rec<MC>& y) {  // RTimesOp
#pragma unroll
  for (int e = 0; e < N; e++) {
    const float pr = rmul(at, b[e].re), pi = rmul(at, b[e].im);
    switch (eqop) {
      case EQ: y[e].re = pr; y[e].im = pi; break;
      case EQM: y[e].re = -pr; y[e].im = -pi; break;
      case PEQ: y[e].re = radd(y[e].re, pr); y[e].im = radd(y[e].im, pi); break;
      default: y[e].re = rsub(y[e].re, pr); y[e].im = rsub(y[e].im, pi); break;
    }
  }
}
template <int N, int MC>
__device__ __forceinline__ void copy_n(int eqop, const Rec<MC>& b, Rec<MC>& y) {  // CopyOp
#pragma unroll
  for (int e = 0; e < N; e++) {
    switch (eqop) {
      case EQ: y[e] = b[e]; break;
      case EQM: y[e].re = -b[e].re; y[e].im = -b[e].im; break;
      case PEQ: y[e].re = radd(y[e].re, b[e].re); y[e].im = radd(y[e].im, b[e].im); break;
      default: y[e].re = rsub(y[e].re, b[e].re); y[e].im = rsub(y[e].im, b[e].im); break;
    }
  }
}

template <int MC>
__device__ __forceinline__ void exec_step(const BStep& S, const Rec<MC>& xa, const Rec<MC>& xb, Rec<MC>& y) {
  const bool load = (S.eqop == PEQ || S.eqop == MEQ);
  switch (S.op) {
    case BOP_LMULT:
      switch (S.kind_b * 4 + S.adja * 2 + S.adjb) {
        case BK_V * 4 + 0: lmult_site<float, 3, 1, false, false>(S.eqop, load, xa, xb, y); break;
        case BK_V * 4 + 2: lmult_site<float, 3, 1, true, false>(S.eqop, load, xa, xb, y); break;
        case BK_H * 4 + 0: lmult_site<float, 3, 2, false, false>(S.eqop, load, xa, xb, y); break;
        case BK_H * 4 + 2: lmult_site<float, 3, 2, true, false>(S.eqop, load, xa, xb, y); break;
        case BK_M * 4 + 0: lmult_site<float, 3, 3, false, false>(S.eqop, load, xa, xb, y); break;
        case BK_M * 4 + 1: lmult_site<float, 3, 3, false, true>(S.eqop, load, xa, xb, y); break;
        case BK_M * 4 + 2: lmult_site<float, 3, 3, true, false>(S.eqop, load, xa, xb, y); break;
        case BK_M * 4 + 3: lmult_site<float, 3, 3, true, true>(S.eqop, load, xa, xb, y); break;
        default:
          if constexpr (MC >= 12) {
            if (S.adja)
              lmult_site<float, 3, 4, true, false>(S.eqop, load, xa, xb, y);
            else
              lmult_site<float, 3, 4, false, false>(S.eqop, load, xa, xb, y);
          }
          break;
      }
      break;
    case BOP_SPPROJ:
      if constexpr (MC >= 12) mu_sign_dispatch<SpprojOp<float, 3>::Body>(S.mu, S.sign, S.eqop, xa, y);
      break;
    case BOP_SPRECON:
      if constexpr (MC >= 12) mu_sign_dispatch<SpreconOp<float, 3>::Body>(S.mu, S.sign, S.eqop, xa, y);
      break;
    case BOP_RTIMES:
      switch (S.kind_r) {
        case BK_V: rtimes_n<3>(S.eqop, S.r, xa, y); break;
        case BK_H: rtimes_n<6>(S.eqop, S.r, xa, y); break;
        case BK_M: rtimes_n<9>(S.eqop, S.r, xa, y); break;
        default:
          if constexpr (MC >= 12) rtimes_n<12>(S.eqop, S.r, xa, y);
          break;
      }
      break;
    default:
      switch (S.kind_r) {
        case BK_V: copy_n<3>(S.eqop, xa, y); break;
        case BK_H: copy_n<6>(S.eqop, xa, y); break;
        case BK_M: copy_n<9>(S.eqop, xa, y); break;
        default:
          if constexpr (MC >= 12) copy_n<12>(S.eqop, xa, y);
          break;
      }
      break;
  }
}

// stored result y of stream S: into the warp's output slice (out != nullptr,
// lane `lane`) or straight to global memory (site i)
template <int MC>
__device__ __forceinline__ void put(const BStream& S, const Rec<MC>& y, unsigned char* out, int lane, long long i) {
  switch (S.kind) {
    case BK_V:
      if (out) st_smem<3>(out + S.out_off + (unsigned)lane * 24u, y); else st_global<3>(S.base + i * 24, y);
      break;
    case BK_H:
      if (out) st_smem<6>(out + S.out_off + (unsigned)lane * 48u, y); else st_global<6>(S.base + i * 48, y);
      break;
    case BK_M:
      if (out) st_smem<9>(out + S.out_off + (unsigned)lane * 72u, y); else st_global<9>(S.base + i * 72, y);
      break;
    default:
      if constexpr (MC >= 12) {
        if (out) st_smem<12>(out + S.out_off + (unsigned)lane * 96u, y); else st_global<12>(S.base + i * 96, y);
      }
      break;
  }
}

// One site through the field's whole program (the generic interpreter).
template <int MC>
__device__ __forceinline__ void run_program_generic(const BField& F, const SiteSrc& src, unsigned char* out,
                                                    int lane) {
  const int ns = F.nsteps;
  Rec<MC> prev;
  int prev_reg = -1;
  for (int k = 0; k < ns; k++) {
    const BStep S = F.st[k];  // uniform across the warp
    Rec<MC> xa, xb, y;
    fetch(xa, S.a, S.kind_a, F, src, prev, prev_reg);
    if (S.op == BOP_LMULT) fetch(xb, S.b, S.kind_b, F, src, prev, prev_reg);
    if (S.eqop == PEQ || S.eqop == MEQ)
      fetch(y, S.load_stream >= 0 ? S.load_stream : S.dst, S.kind_r, F, src, prev, prev_reg);
    exec_step(S, xa, xb, y);
    if (S.spill) set_reg(src, S.dst - kReg0, S.kind_r, y);  // a later, non-adjacent step reads it
    if (S.store >= 0) put(F.s[S.store], y, out, lane, src.i);
    copy_rec(prev, y);
    prev_reg = S.dst;
  }
}

// ---------------------------------------------------------------------------
// Compiled program shapes.  A shape fixes each step's operation, operand
// kinds and adjoints at compile time; a plan whose fields all share one
// shape of the catalogue below runs a kernel instantiated for it: the steps
// are unrolled, every record has its exact length and no step is decoded.
// Operand streams and registers, eqops, mu / sign and the scalar stay
// run-time values of the field's descriptor, and the per-site arithmetic is
// the same as the interpreter's (bit-identical results).
// where a step's operand comes from (classified by the planner)
enum SrcKind : int { SRC_CONTIG = 0, SRC_GATHER = 1, SRC_INOUT = 2, SRC_PREV = 3, SRC_REG = 4, SRC_NONE = 5 };
template <int OP, int KA, int KB, int ADJA, int ADJB, int SA, int SB, int EQOP = -1>  // EQOP -1: run time
struct StepShape {
  static constexpr int op = OP, ka = KA, kb = KB, adja = ADJA, adjb = ADJB, sa = SA, sb = SB, eqop = EQOP;
  static constexpr int kr = OP == BOP_LMULT ? KB : OP == BOP_SPPROJ ? BK_H : OP == BOP_SPRECON ? BK_D : KA;
};
template <class... S>
struct Shape {
  static constexpr int nsteps = sizeof...(S);
};
struct GenericShape {};

// The operand of a compiled shape's first step that is gathered (1: a, 2: b,
// 0: none) and its record length in complex numbers.
template <class SH>
struct LeadGather {
  static constexpr int which = 0, n = 0;
};
template <class S0, class... R>
struct LeadGather<Shape<S0, R...>> {
  static constexpr int which = S0::sb == SRC_GATHER ? 2 : S0::sa == SRC_GATHER ? 1 : 0;
  static constexpr int n = which == 2 ? kncplx(S0::kb) : which == 1 ? kncplx(S0::ka) : 0;
};

// r = u * u2[nbr], w = r * v                          (config 4)
using ShapeConfig4 = Shape<StepShape<BOP_LMULT, BK_M, BK_M, 0, 0, SRC_CONTIG, SRC_GATHER, EQ>,
                           StepShape<BOP_LMULT, BK_M, BK_V, 0, 0, SRC_PREV, SRC_CONTIG, EQ>>;
// out (eqop) sprecon(U spproj(D[nbr]))                 (one Wilson hop direction)
using ShapeHop = Shape<StepShape<BOP_SPPROJ, BK_D, BK_D, 0, 0, SRC_GATHER, SRC_NONE>,
                       StepShape<BOP_LMULT, BK_M, BK_H, 0, 0, SRC_CONTIG, SRC_PREV>,
                       StepShape<BOP_SPRECON, BK_H, BK_H, 0, 0, SRC_PREV, SRC_NONE>>;
// y (eqop) r x, w = U^+ y
using ShapeAxpyMaD = Shape<StepShape<BOP_RTIMES, BK_D, BK_D, 0, 0, SRC_CONTIG, SRC_NONE>,
                           StepShape<BOP_LMULT, BK_M, BK_D, 1, 0, SRC_CONTIG, SRC_PREV>>;
// R = U U2^+, Q (eqop) R
using ShapeMMaCopy = Shape<StepShape<BOP_LMULT, BK_M, BK_M, 0, 1, SRC_CONTIG, SRC_CONTIG>,
                           StepShape<BOP_COPY, BK_M, BK_M, 0, 0, SRC_PREV, SRC_NONE>>;
enum ShapeId : int { SH_GENERIC = 0, SH_CONFIG4 = 1, SH_HOP = 2, SH_AXPY_MAD = 3, SH_MMA_COPY = 4, SH_MULTI = 5 };

template <class SS, int MC>
__device__ __forceinline__ void exec_shaped(const BStep& S, const Rec<MC>& xa, const Rec<MC>& xb, Rec<MC>& y) {
  const bool load = (S.eqop == PEQ || S.eqop == MEQ);
  constexpr int NR = kncplx(SS::kr);
  if constexpr (SS::op == BOP_LMULT) {
    constexpr int NCOL = SS::kb == BK_V ? 1 : SS::kb == BK_H ? 2 : SS::kb == BK_D ? 4 : 3;
    lmult_site<float, 3, NCOL, SS::adja != 0, SS::adjb != 0>(S.eqop, load, xa, xb, y);
  } else if constexpr (SS::op == BOP_SPPROJ) {
    mu_sign_dispatch<SpprojOp<float, 3>::Body>(S.mu, S.sign, S.eqop, xa, y);
  } else if constexpr (SS::op == BOP_SPRECON) {
    mu_sign_dispatch<SpreconOp<float, 3>::Body>(S.mu, S.sign, S.eqop, xa, y);
  } else if constexpr (SS::op == BOP_RTIMES) {
    rtimes_n<NR>(S.eqop, S.r, xa, y);
  } else {
    copy_n<NR>(S.eqop, xa, y);
  }
}

template <int N, int MC>
__device__ __forceinline__ void put_n(const BStream& S, const Rec<MC>& y, unsigned char* out, int lane, long long i) {
  if (out)
    st_smem<N>(out + S.out_off + (unsigned)lane * (N * 8), y);
  else
    st_global<N>(S.base + i * (N * 8), y);
}

// operand `ref` of compile-time source SRC and length N
template <int SRC, int N, int MC>
__device__ __forceinline__ void fetch_src(Rec<MC>& x, int ref, const BField& F, const SiteSrc& src,
                                          const Rec<MC>& prev) {
  if constexpr (SRC == SRC_PREV) {
    copy_rec_n<N>(x, prev);
  } else if constexpr (SRC == SRC_REG) {
    reg_load<N>(x, src, ref - kReg0);
  } else if constexpr (SRC == SRC_GATHER) {
    const BStream& S = F.s[ref];
    long long j = src.stage ? reinterpret_cast<const int*>(src.stage + S.stage_off)[src.t] : S.idx[src.i];
    if (S.nsrc > 0 && (j < 0 || j >= S.nsrc)) {
      raise_dev_error(src.err, QLA_DEVERR_BAD_INDEX);
      zero_rec(x);
    } else {
      ld_global<N>(x, S.base + j * (long long)(N * 8));
    }
  } else {  // SRC_CONTIG, SRC_INOUT
    const BStream& S = F.s[ref];
    if (src.stage)
      ld_smem<N>(x, src.stage + S.stage_off + (unsigned)src.t * (N * 8));
    else if constexpr (SRC == SRC_INOUT)
      ld_global_rw<N>(x, S.base + src.i * (N * 8));
    else
      ld_global<N>(x, S.base + src.i * (N * 8));
  }
}

template <int MC, int K, class SS, class... Rest>
__device__ __forceinline__ void run_shaped(const BField& F, const SiteSrc& src, unsigned char* out, int lane,
                                           Rec<MC>& prev, int prev_reg) {
  BStep S = F.st[K];
  if constexpr (SS::eqop >= 0) S.eqop = SS::eqop;  // a compiled eqop (the planner matched it)
  constexpr int NA = kncplx(SS::ka), NB = kncplx(SS::kb), NR = kncplx(SS::kr);
  Rec<MC> xa, xb, y;
  fetch_src<SS::sa, NA>(xa, S.a, F, src, prev);
  if constexpr (SS::op == BOP_LMULT) fetch_src<SS::sb, NB>(xb, S.b, F, src, prev);
  if (S.eqop == PEQ || S.eqop == MEQ) fetch_n<NR>(y, S.load_stream >= 0 ? S.load_stream : S.dst, F, src, prev, prev_reg);
  exec_shaped<SS>(S, xa, xb, y);
  if (S.spill) reg_store<NR>(src, S.dst - kReg0, y);
  if (S.store >= 0) put_n<NR>(F.s[S.store], y, out, lane, src.i);
  if constexpr (sizeof...(Rest) > 0) {
    copy_rec_n<NR>(prev, y);
    run_shaped<MC, K + 1, Rest...>(F, src, out, lane, prev, S.dst);
  }
}
template <int MC, class... SS>
__device__ __forceinline__ void run_shape(Shape<SS...>, const BField& F, const SiteSrc& src, unsigned char* out,
                                          int lane) {
  Rec<MC> prev;
  run_shaped<MC, 0, SS...>(F, src, out, lane, prev, -1);
}

// A plan whose fields all have catalogue shapes, but not one shape, runs the
// multi-shape kernel: each field's compiled path, chosen per tile (uniform).
// Other plans run the interpreter.
struct MultiShape {};
template <int MC, class SH>
__device__ __forceinline__ void run_program(const BField& F, const SiteSrc& src, unsigned char* out, int lane) {
  if constexpr (std::is_same<SH, GenericShape>::value) {
    run_program_generic<MC>(F, src, out, lane);
  } else if constexpr (std::is_same<SH, MultiShape>::value) {
    switch (F.shape) {
      case SH_CONFIG4: run_shape<MC>(ShapeConfig4{}, F, src, out, lane); break;
      case SH_MMA_COPY: run_shape<MC>(ShapeMMaCopy{}, F, src, out, lane); break;
      case SH_HOP:
        if constexpr (MC >= 12) run_shape<MC>(ShapeHop{}, F, src, out, lane);
        break;
      default:
        if constexpr (MC >= 12) run_shape<MC>(ShapeAxpyMaD{}, F, src, out, lane);
        break;
    }
  } else {
    run_shape<MC>(SH{}, F, src, out, lane);
  }
}

// Copy of field f's descriptor in this warp's shared slot (all lanes take
// part; the caller's lanes then read it from shared memory, not global), kept
// while consecutive tiles belong to the same field.
constexpr int kDescWords = (int)((sizeof(BField) + 15) / 16);  // 16-B words
__device__ __forceinline__ const BField& cached_field(const BatchParams& p, int f, int& cached, uint4* slot,
                                                      int lane) {
  if (f != cached) {
    __syncwarp();  // every lane is done with the previous field's descriptor
    const uint4* src = reinterpret_cast<const uint4*>(p.fields + f);
    for (int w = lane; w < kDescWords; w += 32) slot[w] = __ldg(src + w);
    __syncwarp();
    cached = f;
  }
  return *reinterpret_cast<const BField*>(slot);
}
// the same for the producer, a single lane
__device__ __forceinline__ const BField& cached_field_1(const BatchParams& p, int f, int& cached, uint4* slot) {
  if (f != cached) {
    const uint4* src = reinterpret_cast<const uint4*>(p.fields + f);
    for (int w = 0; w < kDescWords; w++) slot[w] = __ldg(src + w);
    cached = f;
  }
  return *reinterpret_cast<const BField*>(slot);
}

// Dynamic smem: [full[8], empty[8] | abort | tile0 table (8 KB) | S stages |
//               NW output slices | step registers (only when some
//               program spills one): 2 x 12 complex x T | (NW + 1) field
//               descriptors]
// 128 consumer threads (or 64) and one producer warp.  Blocks per SM (the
// register budget each instance compiles to without spilling): a compiled
// shape four (V / H / M records, <= 96 registers) or three (DiracFermions,
// <= 128); the interpreter and the multi-shape kernel three (V / H / M) or
// two (DiracFermions).
constexpr int kBatchThreadsMax = 160;
template <int MC, class SH>
constexpr int batch_min_blocks() {
  constexpr bool compiled = !std::is_same<SH, GenericShape>::value && !std::is_same<SH, MultiShape>::value;
  // (the multi-shape kernel at 12 complex numbers: three blocks with spills
  // measured 0.39 of HBM on a config-4 / hop mix, two 0.38, one at 254
  // registers 0.32)
  constexpr bool multi = std::is_same<SH, MultiShape>::value;
  return MC == 9 ? (compiled ? 4 : 3) : (compiled || multi ? 3 : 2);
}
template <int MC, class SH>
__global__ void __launch_bounds__(kBatchThreadsMax, batch_min_blocks<MC, SH>()) batch_program_kernel(
    const BatchParams p) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int S = p.stages;
  const int NW = (blockDim.x >> 5) - 1;
  const int T = NW * 32;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + 8;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + 128);
  long long* tile0 = reinterpret_cast<long long*>(smem + 256);
  unsigned char* stages = smem + 256 + 8 * kMaxFields;
  unsigned char* outbuf = stages + (size_t)S * p.stage_bytes;
  unsigned char* regs = outbuf + (size_t)NW * p.out_slice_bytes;  // 2 x 12 complex per thread, if needed
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // Tiles are dealt to the blocks in groups of p.chunk consecutive tiles,
  // round-robin: consecutive tiles of a block then mostly belong to one
  // field, so that a warp seldom reloads its cached field descriptor (tiles
  // dealt one by one land in a new field nearly every time on small fields).
  // Block b's k-th tile is tile_of(k).
  const long long C = p.chunk, ngroups = (p.ntiles + C - 1) / C;
  long long my = 0;
  if ((long long)blockIdx.x < ngroups) {
    const long long mg = (ngroups - 1 - (long long)blockIdx.x) / gridDim.x + 1;  // groups of this block
    const bool owns_last = (ngroups - 1 - (long long)blockIdx.x) % gridDim.x == 0;
    my = mg * C - (owns_last ? ngroups * C - p.ntiles : 0);
  }
  auto tile_of = [&](long long k) { return ((long long)blockIdx.x + (k / C) * gridDim.x) * C + k % C; };
  uint4* desc = reinterpret_cast<uint4*>(regs + (p.spill_regs ? (size_t)2 * 12 * 8 * T : 0)) + (size_t)warp * kDescWords;
  int cached = -1;

  for (int f = tid; f < p.nfields; f += blockDim.x) tile0[f] = p.fields[f].tile0;
  if (tid == 0) {
    for (int s = 0; s < S; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], (unsigned)NW);
    }
    *abort_flag = 0;
    mbar_init_fence();
  }
  __syncthreads();
  long long issued = 0;

  if (warp == NW) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      const uint64_t pol = policy_evict_first();
      long long k = 0, round = 0;
      int s = 0;
      for (; k < my; k++) {
        if (round > 0 && !mbar_wait_bounded(&empty[s], (uint32_t)((round - 1) & 1), p.err, 2000000000ull,
                                            abort_flag)) {
          *abort_flag = 1;
          break;
        }
        const long long g = tile_of(k);
        const BField& F = cached_field_1(p, field_of(tile0, p.nfields, g, cached), cached, desc);
        const long long site0 = (g - F.tile0) * T;
        unsigned char* st = stages + (size_t)s * p.stage_bytes;
        if (!F.direct && site0 + T <= F.n) {
          mbar_arrive_expect_tx(&full[s], F.tx_bytes);
          for (int j = 0; j < F.nstreams; j++) {
            const BStream& B = F.s[j];
            const unsigned rb = (unsigned)kncplx(B.kind) * 8u;
            if (B.role == BR_IN && B.idx)
              bulk_g2s(st + B.stage_off, B.idx + site0, (unsigned)T * 4u, &full[s], pol);
            else if (B.role != BR_OUT)
              bulk_g2s(st + B.stage_off, B.base + site0 * rb, (unsigned)T * rb, &full[s], pol);
          }
        } else {
          mbar_arrive(&full[s]);  // partial / unaligned tile: consumers use plain loads
        }
        if (++s == S) {
          s = 0;
          round++;
        }
      }
      issued = k;
    }
  } else {
    // ------------------------------------------------------------ consumers
    const uint64_t pol = policy_evict_first();
    unsigned char* myout = outbuf + (size_t)warp * p.out_slice_bytes;
    int s = 0;
    uint32_t par = 0;
    for (long long k = 0; k < my; k++) {
      if (!mbar_wait_bounded(&full[s], par, p.err, 2000000000ull, abort_flag)) {
        *abort_flag = 1;
        break;
      }
      const long long g = tile_of(k);
      const BField& F = cached_field(p, field_of(tile0, p.nfields, g, cached), cached, desc, lane);
      const long long site0 = (g - F.tile0) * T;
      const int t = warp * 32 + lane;
      const long long i = site0 + t;
      // staged: a full tile of a 16-B aligned field, in the stage; else the
      // same program with plain loads and stores (partial / unaligned tiles)
      const bool staged = !F.direct && site0 + T <= F.n;
      // a compiled shape that starts with a gather: when the block's next tile
      // is the next tile of this field, load this lane's index of it now and
      // prefetch its gathered record into L2 after this tile's arithmetic
      int pf_j = -1;
      if constexpr (LeadGather<SH>::which != 0) {
        if (k + 1 < my && tile_of(k + 1) == g + 1 && i + T < F.n) {
          const BStream& G = F.s[LeadGather<SH>::which == 2 ? F.st[0].b : F.st[0].a];
          pf_j = __ldg(G.idx + i + T);
        }
      }
      unsigned char* ob = myout;
      if (staged) {
        if (lane == 0) bulk_wait_read<0>();  // the slice is no longer read by this warp's previous store
        __syncwarp();
      } else {
        release_stage(&empty[s], lane);  // this warp is done with the stage
      }
      if (staged || i < F.n)  // one call site: the program is inlined once
        run_program<MC, SH>(F, SiteSrc{staged ? stages + (size_t)s * p.stage_bytes : nullptr, t, i, p.err, regs, T},
                            staged ? ob : nullptr, lane);
      if constexpr (LeadGather<SH>::which != 0) {
        const BStream& G = F.s[LeadGather<SH>::which == 2 ? F.st[0].b : F.st[0].a];
        if (pf_j >= 0 && (G.nsrc <= 0 || pf_j < G.nsrc)) {  // only an index the gather would dereference
          constexpr long long RBG = LeadGather<SH>::n * 8;
          const char* q = G.base + (long long)pf_j * RBG;
          prefetch_l2(q);
          prefetch_l2(q + RBG - 8);
        }
      }
      if (staged) {
        // every lane orders its reads of the stage and its writes of the
        // slice before the async proxy: the slice's bulk stores below, and
        // the producer's next bulk copy into the stage released here
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&empty[s]);  // this warp is done with the stage
          const long long s0 = site0 + warp * 32;
          for (int j = 0; j < F.nstreams; j++) {
            const BStream& B = F.s[j];
            if (B.role == BR_IN) continue;
            const unsigned rb = (unsigned)kncplx(B.kind) * 8u;
            bulk_s2g(B.base + s0 * rb, ob + B.out_off, 32u * rb, pol);
          }
          bulk_commit();
        }
      } else if (lane == 0) {
        bulk_commit();  // an empty group keeps the slice bookkeeping aligned
      }
      if (++s == S) {
        s = 0;
        par ^= 1u;
      }
    }
    if (lane == 0) bulk_wait_all<0>();
  }
  __syncthreads();
  if (*abort_flag && warp == NW && lane == 0) {
    // a wait failed: wait (bounded) for every load still in flight before the
    // block's shared memory is released
    for (long long kk = (issued > S ? issued - S : 0); kk < issued; kk++)
      if (!mbar_wait_bounded(&full[kk % S], (uint32_t)((kk / S) & 1), p.err, 200000000ull, nullptr))
        raise_dev_error(p.err, QLA_DEVERR_BULK_TIMEOUT);
  }
}

// ---------------------------------------------------------------------------
// host side: validation, stage layout, plan

static bool plan_error(const char* who, int f, int k, const char* what) {
  char msg[160];
  if (k >= 0)
    std::snprintf(msg, sizeof msg, "field %d, step %d: %s", f, k, what);
  else
    std::snprintf(msg, sizeof msg, "field %d: %s", f, what);
  set_error(QLAGPU_ERR_ARG, who, msg);
  return false;
}

static bool aligned(const void* p, unsigned a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; }

// Checks one program and fills its device descriptor (kinds, stage offsets
// for a tile of T sites, output slice offsets).  Returns false with the
// sticky error set when the program is malformed.
static bool build_field(const char* who, int f, const qlagpu_F3_batch_program& q, int T, BField& b,
                        unsigned& stage_bytes, unsigned& out_slice_bytes, bool& spills, bool& uses_d) {
  std::memset(&b, 0, sizeof(b));
  if (q.n < 0 || q.nstreams < 0 || q.nstreams > kMaxStreams || q.nsteps < 1 || q.nsteps > kMaxSteps)
    return plan_error(who, f, -1, "need n >= 0, 0..8 streams and 1..8 steps");
  b.nstreams = q.nstreams;
  b.nsteps = q.nsteps;
  b.n = q.n;
  bool al16 = true;
  unsigned off = 0, oo = 0;
  for (int j = 0; j < q.nstreams; j++) {
    const qlagpu_batch_stream& s = q.stream[j];
    BStream& d = b.s[j];
    if (s.kind < 0 || s.kind > 3 || s.role < 0 || s.role > 2)
      return plan_error(who, f, -1, "stream kind or role out of range");
    if (!s.base && q.n > 0) return plan_error(who, f, -1, "NULL stream base");
    if (s.index && s.role != BR_IN) return plan_error(who, f, -1, "only IN streams may gather through an index");
    if (s.index && s.nsrc < 0) return plan_error(who, f, -1, "nsrc < 0");
    if (!aligned(s.base, 8) || (s.index && !aligned(s.index, 4)))
      return plan_error(who, f, -1, "stream base must be 8-B aligned and an index 4-B aligned");
    d.base = static_cast<char*>(s.base);
    d.idx = s.index;
    d.nsrc = s.index ? s.nsrc : 0;
    d.kind = s.kind;
    d.role = s.role;
    const unsigned rb = (unsigned)kncplx(s.kind) * 8u;
    if (s.role == BR_IN && s.index) {
      d.stage_off = off;
      off += ((unsigned)T * 4u + 15u) & ~15u;
      b.tx_bytes += (unsigned)T * 4u;
      al16 = al16 && aligned(s.index, 16);
    } else if (s.role != BR_OUT) {
      d.stage_off = off;
      off += ((unsigned)T * rb + 15u) & ~15u;
      b.tx_bytes += (unsigned)T * rb;
    }
    if (!s.index || s.role != BR_IN) al16 = al16 && aligned(s.base, 16);
    if (s.role != BR_IN) {
      d.out_off = oo;
      oo += 32u * rb;
    }
  }
  b.direct = al16 ? 0 : 1;
  int regkind[2] = {-1, -1};
  bool stored[kMaxStreams] = {false};
  auto opnd_kind = [&](int ref, int& kind) -> const char* {
    if (ref == kReg0 || ref == kReg1) {
      kind = regkind[ref - kReg0];
      return kind < 0 ? "operand register read before any step wrote it" : nullptr;
    }
    if (ref < 0 || ref >= q.nstreams) return "operand is neither a stream of the field nor a register";
    if (q.stream[ref].role == BR_OUT) return "operand stream is an output of this launch";
    kind = q.stream[ref].kind;
    return nullptr;
  };
  for (int k = 0; k < q.nsteps; k++) {
    const qlagpu_batch_step& s = q.step[k];
    BStep& d = b.st[k];
    d.op = s.op;
    d.eqop = s.eqop;
    d.a = s.a;
    d.b = s.b;
    d.dst = s.dst;
    d.store = s.store;
    d.adja = s.adja ? 1 : 0;
    d.adjb = s.adjb ? 1 : 0;
    d.mu = s.mu;
    d.sign = s.sign == 1 ? 1 : -1;
    d.r = s.r;
    d.load_stream = -1;
    if (s.op < 0 || s.op > 4) return plan_error(who, f, k, "unknown op");
    if (s.eqop < 0 || s.eqop > 3) return plan_error(who, f, k, "eqop out of range");
    if (s.dst != kReg0 && s.dst != kReg1) return plan_error(who, f, k, "dst must be QLAGPU_REG0 or QLAGPU_REG1");
    if (const char* e = opnd_kind(s.a, d.kind_a)) return plan_error(who, f, k, e);
    switch (s.op) {
      case BOP_LMULT:
        if (d.kind_a != BK_M) return plan_error(who, f, k, "LMULT: a must be a colour matrix");
        if (const char* e = opnd_kind(s.b, d.kind_b)) return plan_error(who, f, k, e);
        if (d.adjb && d.kind_b != BK_M) return plan_error(who, f, k, "LMULT: adjb needs a colour-matrix b");
        d.kind_r = d.kind_b;
        break;
      case BOP_SPPROJ:
        if (d.kind_a != BK_D) return plan_error(who, f, k, "SPPROJ: a must be a DiracFermion");
        if (s.mu < 0 || s.mu > 4) return plan_error(who, f, k, "mu must be 0..4");
        d.kind_r = BK_H;
        break;
      case BOP_SPRECON:
        if (d.kind_a != BK_H) return plan_error(who, f, k, "SPRECON: a must be a HalfFermion");
        if (s.mu < 0 || s.mu > 4) return plan_error(who, f, k, "mu must be 0..4");
        d.kind_r = BK_D;
        break;
      default:
        d.kind_r = d.kind_a;
        break;
    }
    if (s.op != BOP_LMULT) d.kind_b = d.kind_a;
    if (s.store >= 0) {
      if (s.store >= q.nstreams || q.stream[s.store].role == BR_IN)
        return plan_error(who, f, k, "store must name an OUT or INOUT stream");
      if (q.stream[s.store].kind != d.kind_r) return plan_error(who, f, k, "stored stream has another kind");
      if (stored[s.store]) return plan_error(who, f, k, "a stream is stored by more than one step");
      stored[s.store] = true;
    } else if (s.store != -1) {
      return plan_error(who, f, k, "store must be a stream or -1");
    }
    if (s.eqop == PEQ || s.eqop == MEQ) {
      if (s.store >= 0 && q.stream[s.store].role == BR_INOUT) {
        d.load_stream = s.store;
      } else if (regkind[s.dst - kReg0] != d.kind_r) {
        return plan_error(who, f, k, "peq / meq needs an INOUT store stream or a dst register of the result kind");
      }
    }
    regkind[s.dst - kReg0] = d.kind_r;
  }
  for (int j = 0; j < q.nstreams; j++)
    if (q.stream[j].role != BR_IN && !stored[j]) return plan_error(who, f, -1, "an output stream is never stored");
  // register liveness: a register read by a step other than the one right
  // after its writer is also kept in shared memory (the writer spills it)
  for (int k = 0; k < q.nsteps; k++) {
    const BStep& d = b.st[k];
    const int reads[3] = {d.a, d.op == BOP_LMULT ? d.b : -1,
                          ((d.eqop == PEQ || d.eqop == MEQ) && d.load_stream < 0) ? d.dst : -1};
    for (int r : reads) {
      if (r != kReg0 && r != kReg1) continue;
      int w = k - 1;
      while (w >= 0 && b.st[w].dst != r) w--;
      if (w >= 0 && w != k - 1) {
        b.st[w].spill = 1;
        spills = true;
      }
    }
  }
  // operand sources, for matching a compiled shape
  for (int k = 0; k < q.nsteps; k++) {
    BStep& d = b.st[k];
    auto src_of = [&](int ref) {
      if (ref == kReg0 || ref == kReg1) return (k > 0 && b.st[k - 1].dst == ref) ? (int)SRC_PREV : (int)SRC_REG;
      if (q.stream[ref].role == BR_INOUT) return (int)SRC_INOUT;
      return q.stream[ref].index ? (int)SRC_GATHER : (int)SRC_CONTIG;
    };
    d.src_a = src_of(d.a);
    d.src_b = d.op == BOP_LMULT ? src_of(d.b) : (int)SRC_NONE;
  }
  for (int j = 0; j < q.nstreams; j++) uses_d = uses_d || q.stream[j].kind == BK_D;
  for (int k = 0; k < q.nsteps; k++)
    uses_d = uses_d || b.st[k].kind_r == BK_D || b.st[k].kind_a == BK_D || b.st[k].kind_b == BK_D;
  if (off > stage_bytes) stage_bytes = off;
  if (oo > out_slice_bytes) out_slice_bytes = oo;
  return true;
}

// the catalogue shape that every field's program has, or SH_GENERIC
template <class... SS>
static bool has_shape(const BField& b, Shape<SS...>) {
  constexpr int ops[] = {SS::op...}, ka[] = {SS::ka...}, kb[] = {SS::kb...}, aa[] = {SS::adja...},
                ab[] = {SS::adjb...}, sa[] = {SS::sa...}, sb[] = {SS::sb...}, eq[] = {SS::eqop...};
  if (b.nsteps != (int)sizeof...(SS)) return false;
  for (int k = 0; k < b.nsteps; k++) {
    const BStep& d = b.st[k];
    if (d.op != ops[k] || d.kind_a != ka[k] || (d.op == BOP_LMULT && d.kind_b != kb[k]) || d.adja != aa[k] ||
        d.adjb != ab[k] || d.src_a != sa[k] || d.src_b != sb[k] || (eq[k] >= 0 && d.eqop != eq[k]))
      return false;
  }
  return true;
}
static int shape_of(const BField& b) {
  if (has_shape(b, ShapeConfig4{})) return SH_CONFIG4;
  if (has_shape(b, ShapeHop{})) return SH_HOP;
  if (has_shape(b, ShapeAxpyMaD{})) return SH_AXPY_MAD;
  if (has_shape(b, ShapeMMaCopy{})) return SH_MMA_COPY;
  return SH_GENERIC;
}
// sets each field's shape; returns the shape all fields share, SH_MULTI when
// every field has a catalogue shape but not the same one, else SH_GENERIC
static int common_shape(BField* h, int nfields) {
  int common = -1;
  bool all_known = true;
  for (int f = 0; f < nfields; f++) {
    h[f].shape = shape_of(h[f]);
    all_known = all_known && h[f].shape != SH_GENERIC;
    common = (common < 0 || common == h[f].shape) ? h[f].shape : SH_MULTI;
  }
  if (!all_known || common < 0) return SH_GENERIC;
  return common;
}
static const void* batch_kernel_for(const BatchPlan* plan) {
  switch (plan->shape) {
    case SH_CONFIG4: return reinterpret_cast<const void*>(&batch_program_kernel<9, ShapeConfig4>);
    case SH_HOP: return reinterpret_cast<const void*>(&batch_program_kernel<12, ShapeHop>);
    case SH_AXPY_MAD: return reinterpret_cast<const void*>(&batch_program_kernel<12, ShapeAxpyMaD>);
    case SH_MMA_COPY: return reinterpret_cast<const void*>(&batch_program_kernel<9, ShapeMMaCopy>);
    case SH_MULTI:
      return plan->mc == 12 ? reinterpret_cast<const void*>(&batch_program_kernel<12, MultiShape>)
                            : reinterpret_cast<const void*>(&batch_program_kernel<9, MultiShape>);
    default:
      return plan->mc == 12 ? reinterpret_cast<const void*>(&batch_program_kernel<12, GenericShape>)
                            : reinterpret_cast<const void*>(&batch_program_kernel<9, GenericShape>);
  }
}

static BatchPlan* make_plan(const char* who, const qlagpu_F3_batch_program* fields, int nfields) {
  if (!fields || nfields <= 0 || nfields > kMaxFields) {
    set_error(QLAGPU_ERR_ARG, who, "need 1 <= nfields <= 1024 and a field table");
    return nullptr;
  }
  int t = 128, st = 2;
  if (!tuned_shape("F3_batch_program", &t, &st) || (t != 64 && t != 128)) {
    t = 128;  // the kernel's launch bounds allow 64 or 128 sites per tile
    st = 2;
  }
  std::vector<BField> h((size_t)nfields);
  unsigned stage_bytes = 0, out_slice = 0;
  bool spills = false, uses_d = false;
  long long tiles = 0;
  for (int f = 0; f < nfields; f++) {
    if (!build_field(who, f, fields[f], t, h[(size_t)f], stage_bytes, out_slice, spills, uses_d)) return nullptr;
    h[(size_t)f].tile0 = tiles;
    tiles += (fields[f].n + t - 1) / t;
  }
  stage_bytes = (stage_bytes + 127u) & ~127u;
  if (stage_bytes == 0) stage_bytes = 128;
  out_slice = (out_slice + 127u) & ~127u;
  auto smem_for = [&](int stages) {
    return 256 + 8 * (size_t)kMaxFields + (size_t)stages * stage_bytes + (size_t)(t / 32) * out_slice +
           (spills ? 2 * 12 * 8 * (size_t)t : 0) + 16 * (size_t)kDescWords * (t / 32 + 1);
  };
  size_t smem = smem_for(st);
  while (smem > 225u * 1024u && st > 2) smem = smem_for(--st);  // shed stages before giving up
  if (smem > 225u * 1024u) {
    set_error(QLAGPU_ERR_ARG, who, "the programs' streams need more shared memory per tile than a block has");
    return nullptr;
  }
  const int shape = common_shape(h.data(), nfields);  // also each field's own shape
  if (!device_error_word()) return nullptr;  // allocate it now, not inside a later capture
  BatchPlan* plan = new BatchPlan();
  plan->nfields = nfields;
  plan->ntiles = tiles;
  plan->threads = t;
  plan->stages = st;
  plan->stage_bytes = stage_bytes;
  plan->out_slice_bytes = out_slice;
  plan->spill_regs = spills ? 1 : 0;
  plan->mc = uses_d ? 12 : 9;
  plan->shape = shape;
  plan->smem = smem;
  if (cudaMalloc(&plan->dfields, sizeof(BField) * (size_t)nfields) != cudaSuccess ||
      cudaMemcpy(plan->dfields, h.data(), sizeof(BField) * (size_t)nfields, cudaMemcpyHostToDevice) !=
          cudaSuccess) {
    check_launch(who);
    set_error(QLAGPU_ERR_ALLOC, who, "plan table allocation failed");
    cudaFree(plan->dfields);
    delete plan;
    return nullptr;
  }
  const void* fn = batch_kernel_for(plan);
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plan->smem);
  int nb = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, t + 32, plan->smem) != cudaSuccess || nb < 1) nb = 1;
  cudaGetLastError();
  long long grid = (long long)nb * device_sm_count();
  if (grid > tiles) grid = tiles;
  plan->grid = (int)(grid < 1 ? 1 : grid);
  // Tile groups, measured on B200 (64 uneven fields, fraction of HBM peak by
  // group size 1 / 4 / 8 / 16 / one contiguous run per block): config 4's
  // shape 0.78 / 0.83 / 0.86 / 0.88 / 0.91, where each tile's work is short
  // and a descriptor reload per tile shows; the hop shape 0.67 / 0.72 / 0.73 /
  // 0.72 / 0.74 and a config-4 / hop mix 0.37 / 0.38 / 0.39 / 0.38 / 0.39.
  plan->chunk = shape == SH_CONFIG4 ? (tiles + plan->grid - 1) / plan->grid : 8;
  return plan;
}

}  // namespace qlab

using namespace qlab;

extern "C" QLAB_EXPORT void* qlagpu_F3_batch_plan_program(const qlagpu_F3_batch_program* fields, int nfields) {
  return make_plan("qlagpu_F3_batch_plan_program", fields, nfields);
}

// The fixed sequence r = u * u2[nbr] (QLA_F3_M_eq_M_times_xM), w = r * v
// (QLA_F3_V_veq_M_times_V) as a two-step program per field.
extern "C" QLAB_EXPORT void* qlagpu_F3_batch_plan(const qlagpu_F3_batch_field* fields, int nfields) {
  const char* who = "qlagpu_F3_batch_plan";
  if (!fields || nfields <= 0 || nfields > kMaxFields) {
    set_error(QLAGPU_ERR_ARG, who, "need 1 <= nfields <= 1024 and a field table");
    return nullptr;
  }
  std::vector<qlagpu_F3_batch_program> prog((size_t)nfields);
  for (int f = 0; f < nfields; f++) {
    const qlagpu_F3_batch_field& q = fields[f];
    if (!q.r || !q.u || !q.u2 || !q.nbr || !q.w || !q.v || q.n < 0) {
      set_error(QLAGPU_ERR_NULLPTR, who, "NULL array in a field (or n < 0)");
      return nullptr;
    }
    qlagpu_F3_batch_program& p = prog[(size_t)f];
    std::memset(&p, 0, sizeof(p));
    p.n = q.n;
    p.nstreams = 5;
    p.nsteps = 2;
    p.stream[0] = qlagpu_batch_stream{q.u, nullptr, 0, QLAGPU_REC_M, QLAGPU_STREAM_IN};
    p.stream[1] = qlagpu_batch_stream{q.u2, q.nbr, 0, QLAGPU_REC_M, QLAGPU_STREAM_IN};
    p.stream[2] = qlagpu_batch_stream{q.v, nullptr, 0, QLAGPU_REC_V, QLAGPU_STREAM_IN};
    p.stream[3] = qlagpu_batch_stream{q.r, nullptr, 0, QLAGPU_REC_M, QLAGPU_STREAM_OUT};
    p.stream[4] = qlagpu_batch_stream{q.w, nullptr, 0, QLAGPU_REC_V, QLAGPU_STREAM_OUT};
    p.step[0] = qlagpu_batch_step{QLAGPU_BOP_LMULT, QLAGPU_EQ, 0, 1, QLAGPU_REG0, 3, 0, 0, 0, 1, 0.f};
    p.step[1] = qlagpu_batch_step{QLAGPU_BOP_LMULT, QLAGPU_EQ, QLAGPU_REG0, 2, QLAGPU_REG1, 4, 0, 0, 0, 1, 0.f};
  }
  return make_plan(who, prog.data(), nfields);
}

extern "C" QLAB_EXPORT int qlagpu_batch_run(void* handle) {
  QLAB_TRACE("qlagpu_batch_run");
  BatchPlan* plan = static_cast<BatchPlan*>(handle);
  if (!plan) {
    set_error(QLAGPU_ERR_NULLPTR, "qlagpu_batch_run", "NULL plan");
    return QLAGPU_ERR_NULLPTR;
  }
  if (plan->ntiles == 0) return QLAGPU_OK;
  BatchParams p;
  p.fields = plan->dfields;
  p.nfields = plan->nfields;
  p.ntiles = plan->ntiles;
  p.stages = plan->stages;
  p.stage_bytes = plan->stage_bytes;
  p.out_slice_bytes = plan->out_slice_bytes;
  p.spill_regs = plan->spill_regs;
  p.chunk = plan->chunk;
  p.err = device_error_word();
  void* args[] = {&p};
  const void* fn = batch_kernel_for(plan);
  if (cudaLaunchKernel(fn, dim3((unsigned)plan->grid),
                       dim3((unsigned)plan->threads + 32u), args, plan->smem, current_stream()) != cudaSuccess) {
    check_launch("qlagpu_batch_run");
    return QLAGPU_ERR_LAUNCH;
  }
  return check_launch("qlagpu_batch_run") ? QLAGPU_OK : QLAGPU_ERR_LAUNCH;
}

extern "C" QLAB_EXPORT void qlagpu_batch_destroy(void* handle) {
  BatchPlan* plan = static_cast<BatchPlan*>(handle);
  if (!plan) return;
  cudaFree(plan->dfields);
  delete plan;
}
