// qla_engine.cuh -- the site-loop engine behind every level-1 QLA operator.
//
// QLA's generated functions are loops `for(i<n)` over AoS site records
// (lib/perl/formatting.pl:90-127).  On B200 such a loop is HBM-bound, and
// AoS records of 24/48/72/96 B are awkward for per-thread coalescing.  The
// engine therefore moves whole tiles of T consecutive sites of every
// contiguous operand with 1-D bulk (TMA) copies into shared memory, in an
// S-stage mbarrier pipeline, computes one site per thread from shared memory,
// and writes the destination tile back with one bulk store.  Operands reached
// through a pointer array (`pX`, 8 B per site) or an int32 index stream
// (`xX`, 4 B per site) stream their pointer/index tile through the same
// pipeline and gather the records with per-thread read-only loads.
//
// A second, direct kernel (no staging) runs the gang-index `x` variants, whose
// every operand is scattered, and any call whose pointers are not 16-B
// aligned (bulk copies require 16-B alignment).  Both kernels share the
// per-site code, so their results are identical.
//
// An operator type OP provides:
//   using R;                               site real type (float/double)
//   NIN, N0, N1, N2                        number of inputs, complex numbers per input record
//   NOUT                                   complex numbers per destination record (0 = none)
//   NACC                                   number of double accumulators (0 = not a reduction)
//   apply(p, x0, x1, x2, y)                destination record y (pre-loaded when p.out_read)
//   accum(p, x0, x1, x2, acc)              reduction contribution of one site
#pragma once
#include "qla_core.cuh"

namespace qlab {

enum OpndMode : int { OM_NONE = 0, OM_CONTIG = 1, OM_PTR = 2, OM_IDX = 3 };

struct Opnd {
  const void* base;         // CONTIG / IDX: record array
  const void* const* ptrs;  // PTR: device array of record pointers (one per site)
  const int* idx;           // IDX: int32 record index per site
  int mode;
};

struct SiteParams {
  Opnd in[3];
  void* out;         // destination field (record array)
  int out_read;      // destination is also read (peq / meq)
  const int* gang;   // gang index (x variants): site k = gang[i]
  long long n;       // loop length
  int eqop, mu, sign, aux;
  double sval, sval_im;  // scalar argument passed by value (host scalar)
  const void* sptr;      // scalar argument left on the device (read by the kernel)
  // reductions
  DD* partials;
  unsigned* counter;
  void* result;      // device address receiving the reduced value(s)
  unsigned* err;     // device error word (QLA_DEVERR_* bits)
  // bulk-copy pipeline layout (host-computed)
  unsigned stage_bytes, tx_bytes;
  unsigned off_in[3], off_out_in;
  int stages;        // pipeline depth S (1..8)
  long long ntiles;  // number of full tiles of T sites
};

template <int N>
struct ArrN {
  static constexpr int value = N > 0 ? N : 1;
};

// ---------------------------------------------------------------------------
// per-site work shared by both kernels

template <class OP, int N>
__device__ __forceinline__ void fetch_gathered(Cx<typename OP::R> (&x)[ArrN<N>::value], const Opnd& o, long long k) {
  using R = typename OP::R;
  constexpr int RB = N * (int)sizeof(Cx<R>);
  const void* src;
  if (o.mode == OM_PTR)
    src = o.ptrs[k];
  else if (o.mode == OM_IDX)
    src = static_cast<const char*>(o.base) + (long long)o.idx[k] * RB;
  else
    src = static_cast<const char*>(o.base) + k * RB;
  load_rec_global<R, ArrN<N>::value>(x, src);
}

// Direct path: all operands read straight from global memory for site k.
template <class OP>
__device__ __forceinline__ void site_direct(const SiteParams& p, long long k, double* acc) {
  using R = typename OP::R;
  Cx<R> x0[ArrN<OP::N0>::value], x1[ArrN<OP::N1>::value], x2[ArrN<OP::N2>::value];
  if constexpr (OP::NIN > 0) fetch_gathered<OP, OP::N0>(x0, p.in[0], k);
  if constexpr (OP::NIN > 1) fetch_gathered<OP, OP::N1>(x1, p.in[1], k);
  if constexpr (OP::NIN > 2) fetch_gathered<OP, OP::N2>(x2, p.in[2], k);
  if constexpr (OP::NOUT > 0) {
    constexpr int OB = OP::NOUT * (int)sizeof(Cx<R>);
    char* dst = static_cast<char*>(p.out) + k * OB;
    Cx<R> y[OP::NOUT];
    if (p.out_read) load_rec_rw<R, OP::NOUT>(y, dst);
    OP::apply(p, x0, x1, x2, y);
    store_rec<R, OP::NOUT>(dst, y);
  } else {
    OP::accum(p, x0, x1, x2, acc);
  }
}

// Staged path: contiguous operands come from the shared-memory tile `st`,
// pointer/index operands take their pointer/index from the tile and gather.
template <class OP, int N>
__device__ __forceinline__ void fetch_staged(Cx<typename OP::R> (&x)[ArrN<N>::value], const Opnd& o,
                                             const unsigned char* st, unsigned off, int t) {
  using R = typename OP::R;
  constexpr int RB = N * (int)sizeof(Cx<R>);
  if (o.mode == OM_CONTIG) {
    load_rec<R, ArrN<N>::value>(x, st + off + (unsigned)t * RB);
  } else if (o.mode == OM_PTR) {
    const void* src = reinterpret_cast<const void* const*>(st + off)[t];
    load_rec_global<R, ArrN<N>::value>(x, src);
  } else {
    const int j = reinterpret_cast<const int*>(st + off)[t];
    load_rec_global<R, ArrN<N>::value>(x, static_cast<const char*>(o.base) + (long long)j * RB);
  }
}

// Block-level reduction of NACC double-double accumulators into the
// per-block partial slots, then a last-block-done finish that writes the
// total to p.result.  The summation order depends only on the grid, so
// results are deterministic run to run on a given device.
template <class OP>
__device__ void reduce_finish(const SiteParams& p, DD (&acc)[ArrN<OP::NACC>::value]) {
  constexpr int NA = ArrN<OP::NACC>::value;
  __shared__ DD red[32][NA];
  __shared__ bool is_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int a = 0; a < NA; a++) {
    for (int m = 16; m >= 1; m >>= 1) dd_merge(acc[a], dd_shfl_xor(acc[a], m));
    if (lane == 0) red[warp][a] = acc[a];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int a = 0; a < NA; a++) {
      DD s = red[0][a];
      for (int w = 1; w < nwarps; w++) dd_merge(s, red[w][a]);
      p.partials[(long long)blockIdx.x * NA + a] = s;
    }
    __threadfence();
    unsigned ticket = atomicAdd(p.counter, 1u);
    is_last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  // last block: fold the partials in a fixed order
  DD s[NA];
  for (int a = 0; a < NA; a++) s[a] = DD{0.0, 0.0};
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
    for (int a = 0; a < NA; a++) {
      volatile DD* vp = reinterpret_cast<volatile DD*>(&p.partials[(long long)b * NA + a]);
      DD v;
      v.hi = vp->hi;
      v.lo = vp->lo;
      dd_merge(s[a], v);
    }
  for (int a = 0; a < NA; a++) {
    for (int m = 16; m >= 1; m >>= 1) dd_merge(s[a], dd_shfl_xor(s[a], m));
    if (lane == 0) red[warp][a] = s[a];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot[NA];
    for (int a = 0; a < NA; a++) {
      DD t = red[0][a];
      for (int w = 1; w < nwarps; w++) dd_merge(t, red[w][a]);
      tot[a] = __dadd_rn(t.hi, t.lo);
    }
    OP::finish(p, tot);
    *p.counter = 0u;  // ready for the next launch on this scratch
  }
}

template <class OP>
__device__ __forceinline__ void acc_fold(DD (&dacc)[ArrN<OP::NACC>::value], const double* acc) {
#pragma unroll
  for (int a = 0; a < ArrN<OP::NACC>::value; a++) dd_add(dacc[a], acc[a]);
}

// ---------------------------------------------------------------------------
// Kernel 1: bulk-copy (TMA) pipeline, persistent, warp-specialised.
//
// Block = NW consumer warps (one site per lane per tile, T = 32*NW sites per
// tile) + 1 producer warp.  Per stage s there is a `full` mbarrier (completed
// by the bulk-copy transaction bytes) and an `empty` mbarrier (one arrival
// per consumer warp once it has read the stage).  The producer lane waits on
// `empty`, re-arms `full` and issues the next tile's loads; consumer warps
// wait on `full`, compute, release the stage, and write their 32 results
// through a per-warp double-buffered shared-memory slice with their own bulk
// store.  No block-wide barrier sits in the tile loop, so every warp runs at
// its own pace and the next loads go out as soon as a stage is released.
//
// Dynamic shared memory: [full[S], empty[S], abort flag | S stages |
//                         NW x 2 destination slices of 32 records].
// Every wait is time-bounded; a failed wait raises the abort flag so that all
// other waits of the block give up at once, and loads still in flight are
// drained (bounded) before the block exits.
template <class OP>
__global__ void __launch_bounds__(288) site_tma_kernel(const SiteParams p) {
  using R = typename OP::R;
  constexpr int OB = OP::NOUT * (int)sizeof(Cx<R>);
  constexpr int NA = ArrN<OP::NACC>::value;
  extern __shared__ __align__(128) unsigned char smem[];
  const int S = p.stages;
  const int NW = (blockDim.x >> 5) - 1;  // consumer warps
  const int T = NW * 32;                 // sites per tile
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + 8;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + 8 * 16);
  unsigned char* stages = smem + 256;
  unsigned char* outbuf = stages + (size_t)S * p.stage_bytes;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long my =
      ((long long)blockIdx.x < p.ntiles) ? (p.ntiles - 1 - (long long)blockIdx.x) / gridDim.x + 1 : 0;

  if (tid == 0) {
    for (int s = 0; s < S; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], (unsigned)NW);
    }
    *abort_flag = 0;
    mbar_init_fence();
  }
  __syncthreads();

  DD dacc[NA];
#pragma unroll
  for (int a = 0; a < NA; a++) dacc[a] = DD{0.0, 0.0};
  bool alive = true;
  long long issued = 0;  // tiles whose loads the producer issued

  if (warp == NW) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      const uint64_t pol = policy_evict_first();
      constexpr int RB[3] = {OP::N0 * (int)sizeof(Cx<R>), OP::N1 * (int)sizeof(Cx<R>),
                             OP::N2 * (int)sizeof(Cx<R>)};
      long long k = 0;
      int s = 0;
      long long round = 0;  // k / S
      for (; k < my; k++) {
        // stage s was last filled in round-1; wait until its consumers released it
        if (round > 0 && !mbar_wait_bounded(&empty[s], (uint32_t)((round - 1) & 1), p.err, 2000000000ull,
                                            abort_flag)) {
          *abort_flag = 1;
          break;
        }
        const long long site0 = ((long long)blockIdx.x + k * gridDim.x) * T;
        unsigned char* st = stages + (size_t)s * p.stage_bytes;
        mbar_arrive_expect_tx(&full[s], p.tx_bytes);
#pragma unroll
        for (int j = 0; j < OP::NIN; j++) {
          const Opnd& o = p.in[j];
          if (o.mode == OM_CONTIG)
            bulk_g2s(st + p.off_in[j], static_cast<const char*>(o.base) + site0 * RB[j], (unsigned)T * RB[j],
                     &full[s], pol);
          else if (o.mode == OM_PTR)
            bulk_g2s(st + p.off_in[j], o.ptrs + site0, (unsigned)T * 8u, &full[s], pol);
          else
            bulk_g2s(st + p.off_in[j], o.idx + site0, (unsigned)T * 4u, &full[s], pol);
        }
        if constexpr (OP::NOUT > 0) {
          if (p.out_read)
            bulk_g2s(st + p.off_out_in, static_cast<const char*>(p.out) + site0 * OB, (unsigned)T * OB, &full[s],
                     pol);
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
    unsigned char* myout = outbuf + (size_t)warp * 2 * 32 * OB;
    int s = 0;
    uint32_t par = 0;
    for (long long k = 0; k < my; k++) {
      if (!mbar_wait_bounded(&full[s], par, p.err, 2000000000ull, abort_flag)) {
        *abort_flag = 1;
        alive = false;
        break;
      }
      const unsigned char* st = stages + (size_t)s * p.stage_bytes;
      const int t = warp * 32 + lane;
      Cx<R> x0[ArrN<OP::N0>::value], x1[ArrN<OP::N1>::value], x2[ArrN<OP::N2>::value];
      Cx<R> y[ArrN<OP::NOUT>::value];
      if constexpr (OP::NIN > 0) fetch_staged<OP, OP::N0>(x0, p.in[0], st, p.off_in[0], t);
      if constexpr (OP::NIN > 1) fetch_staged<OP, OP::N1>(x1, p.in[1], st, p.off_in[1], t);
      if constexpr (OP::NIN > 2) fetch_staged<OP, OP::N2>(x2, p.in[2], st, p.off_in[2], t);
      if constexpr (OP::NOUT > 0) {
        if (p.out_read) load_rec<R, OP::NOUT>(y, st + p.off_out_in + (unsigned)t * OB);
      }
      if constexpr (OP::NOUT > 0) {
        OP::apply(p, x0, x1, x2, y);
        unsigned char* ob = myout + (size_t)(k & 1) * 32 * OB;
        if (lane == 0) bulk_wait_read<1>();  // slice (k&1) no longer read by this warp's store k-2
        __syncwarp();
        store_rec_smem<R, OP::NOUT>(ob + (unsigned)lane * OB, y);
        // every lane orders its reads of the stage and its writes of the
        // slice before the async proxy: the slice's bulk store below, and
        // the producer's next bulk copy into the stage released here
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&empty[s]);  // this warp is done with the stage
          const long long site0 = ((long long)blockIdx.x + k * gridDim.x) * T + warp * 32;
          bulk_s2g(static_cast<char*>(p.out) + site0 * OB, ob, 32u * OB, pol);
          bulk_commit();
        }
      } else {
        release_stage(&empty[s], lane);  // this warp is done with the stage
        double acc[NA];
        OP::accum(p, x0, x1, x2, acc);
        acc_fold<OP>(dacc, acc);
      }
      if (++s == S) {
        s = 0;
        par ^= 1u;
      }
    }
    if constexpr (OP::NOUT > 0) {
      if (lane == 0) bulk_wait_all<0>();
    }
    // partial last tile: plain loads by the consumers of the last block
    if (alive && blockIdx.x == gridDim.x - 1) {
      const long long k0 = p.ntiles * T + warp * 32 + lane;
      if (k0 < p.n) {
        double acc[NA];
        site_direct<OP>(p, k0, acc);
        if constexpr (OP::NACC > 0) acc_fold<OP>(dacc, acc);
      }
    }
  }
  __syncthreads();
  if (*abort_flag && warp == NW && lane == 0) {
    // a wait failed: before the block's shared memory is released, wait
    // (bounded) until every load still in flight has landed
    for (long long kk = (issued > S ? issued - S : 0); kk < issued; kk++)
      if (!mbar_wait_bounded(&full[kk % S], (uint32_t)((kk / S) & 1), p.err, 200000000ull, nullptr))
        raise_dev_error(p.err, QLA_DEVERR_BULK_TIMEOUT);
  }
  // every block takes part in the finish, even after a failed wait, so that
  // the ticket counter returns to zero (the error word marks the result invalid)
  if constexpr (OP::NACC > 0) reduce_finish<OP>(p, dacc);
}

// ---------------------------------------------------------------------------
// Kernel 2: direct, grid-stride, one site per thread (gang-index variants and
// unaligned operands).
template <class OP>
__global__ void __launch_bounds__(256) site_direct_kernel(const SiteParams p) {
  constexpr int NA = ArrN<OP::NACC>::value;
  DD dacc[NA];
#pragma unroll
  for (int a = 0; a < NA; a++) dacc[a] = DD{0.0, 0.0};
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += stride) {
    const long long k = p.gang ? (long long)p.gang[i] : i;
    double acc[NA];
    site_direct<OP>(p, k, acc);
    if constexpr (OP::NACC > 0) acc_fold<OP>(dacc, acc);
  }
  if constexpr (OP::NACC > 0) reduce_finish<OP>(p, dacc);
}

}  // namespace qlab
