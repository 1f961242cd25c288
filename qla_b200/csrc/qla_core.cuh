// qla_core.cuh -- device-side building blocks shared by every QLA B200 kernel.
//
//  * complex arithmetic that restates the QLA complex macros
//    (include/qla_complex.h:147-405) with explicitly rounded operations
//    (__fmul_rn/__fadd_rn/... never contract into FMA), so that site results
//    are bit-identical to the reference's C compiled on x86-64;
//  * record load/store helpers for the AoS site records
//    (include/qla_types.h:29-33: V[nc], H[nc][2], D[nc][4], M[nc][nc]);
//  * thin inline-PTX wrappers for sm_100a mbarriers and bulk (1-D TMA)
//    copies, with time-bounded waits that record an error instead of hanging.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace qlab {

// ---------------------------------------------------------------------------
// error bits written by kernels into the device error word (read by the host
// through qlagpu_device_error()).
enum : unsigned {
  QLA_DEVERR_MBAR_TIMEOUT = 1u,   // an mbarrier wait gave up
  QLA_DEVERR_BULK_TIMEOUT = 2u,   // draining in-flight bulk copies gave up
  QLA_DEVERR_BAD_INDEX = 4u,      // an index stream entry was out of range
  QLA_DEVERR_MFUNC_NOCONV = 8u,   // an iterative matrix function hit its cap
  QLA_DEVERR_RNG = 16u,           // the polar gaussian's rejection loop hit its cap
};

// The error word lives in device memory owned by the runtime (one per
// device); kernels receive its address with their parameters.
__device__ __forceinline__ void raise_dev_error(unsigned* err, unsigned bits) {
  if (err) atomicOr(err, bits);
}

// ---------------------------------------------------------------------------
// explicitly rounded scalar arithmetic (no FMA contraction)
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double rdiv(double a, double b) { return __ddiv_rn(a, b); }

template <typename R>
struct Cx {
  R re, im;
};

// eqop codes shared with the host: eq, peq, meq, eqm
enum Eqop : int { EQ = 0, PEQ = 1, MEQ = 2, EQM = 3 };

// x (+|-)= a*b with the conjugation pattern (ca, cb); restates
// qla_complex.h:330-333 (c_peq_c_times_c), 386-389 (ca_times_c),
// 366-369 (c_times_ca), 347-350 (ca_times_ca) and their meq forms.
template <bool CA, bool CB, typename R>
__device__ __forceinline__ void cmac(Cx<R>& x, bool minus, Cx<R> a, Cx<R> b) {
  R re, im;
  if (!CA && !CB) {
    re = rsub(rmul(a.re, b.re), rmul(a.im, b.im));
    im = radd(rmul(a.re, b.im), rmul(a.im, b.re));
  } else if (CA && !CB) {
    re = radd(rmul(a.re, b.re), rmul(a.im, b.im));
    im = rsub(rmul(a.re, b.im), rmul(a.im, b.re));
  } else if (!CA && CB) {
    re = radd(rmul(a.re, b.re), rmul(a.im, b.im));
    im = rsub(rmul(a.im, b.re), rmul(a.re, b.im));
  } else {
    re = rsub(rmul(a.re, b.re), rmul(a.im, b.im));
    im = rsub(rmul(-a.re, b.im), rmul(a.im, b.re));
  }
  if (minus) {
    x.re = rsub(x.re, re);
    x.im = rsub(x.im, im);
  } else {
    x.re = radd(x.re, re);
    x.im = radd(x.im, im);
  }
}

// ---------------------------------------------------------------------------
// record movement.  A record of N complex numbers of type R lives at an
// address aligned to sizeof(Cx<R>) (8 B for float, 16 B for double).
template <typename R, int N>
__device__ __forceinline__ void load_rec(Cx<R> (&x)[N], const void* p) {
  if constexpr (sizeof(R) == 4 && (N % 2) == 0) {
    // records of a multiple of 16 B (H, D) start 16-B aligned in a staged
    // tile: 16-B accesses halve the shared-memory bank conflicts of the
    // 48/96-B record stride
    const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
    for (int e = 0; e < N / 2; e++) {
      float4 v = q[e];
      x[2 * e].re = v.x;
      x[2 * e].im = v.y;
      x[2 * e + 1].re = v.z;
      x[2 * e + 1].im = v.w;
    }
  } else if constexpr (sizeof(R) == 4) {
    const float2* q = reinterpret_cast<const float2*>(p);
#pragma unroll
    for (int e = 0; e < N; e++) {
      float2 v = q[e];
      x[e].re = v.x;
      x[e].im = v.y;
    }
  } else {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int e = 0; e < N; e++) {
      double2 v = q[e];
      x[e].re = v.x;
      x[e].im = v.y;
    }
  }
}

// shared-memory store of a record; same vector width rule as load_rec
template <typename R, int N>
__device__ __forceinline__ void store_rec_smem(void* p, const Cx<R> (&x)[N]) {
  if constexpr (sizeof(R) == 4 && (N % 2) == 0) {
    float4* q = reinterpret_cast<float4*>(p);
#pragma unroll
    for (int e = 0; e < N / 2; e++) q[e] = make_float4(x[2 * e].re, x[2 * e].im, x[2 * e + 1].re, x[2 * e + 1].im);
  } else if constexpr (sizeof(R) == 4) {
    float2* q = reinterpret_cast<float2*>(p);
#pragma unroll
    for (int e = 0; e < N; e++) q[e] = make_float2(x[e].re, x[e].im);
  } else {
    double2* q = reinterpret_cast<double2*>(p);
#pragma unroll
    for (int e = 0; e < N; e++) q[e] = make_double2(x[e].re, x[e].im);
  }
}

// read-only global load (the input fields are never written by the kernel)
template <typename R, int N>
__device__ __forceinline__ void load_rec_global(Cx<R> (&x)[N], const void* p) {
  if constexpr (sizeof(R) == 4) {
    const float2* q = reinterpret_cast<const float2*>(p);
#pragma unroll
    for (int e = 0; e < N; e++) {
      float2 v = __ldg(q + e);
      x[e].re = v.x;
      x[e].im = v.y;
    }
  } else {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int e = 0; e < N; e++) {
      double2 v = __ldg(q + e);
      x[e].re = v.x;
      x[e].im = v.y;
    }
  }
}

// plain global load (used where the record may alias the output, i.e. the
// destination of a peq/meq update)
template <typename R, int N>
__device__ __forceinline__ void load_rec_rw(Cx<R> (&x)[N], const void* p) {
  if constexpr (sizeof(R) == 4) {
    const float2* q = reinterpret_cast<const float2*>(p);
#pragma unroll
    for (int e = 0; e < N; e++) {
      float2 v = q[e];
      x[e].re = v.x;
      x[e].im = v.y;
    }
  } else {
    load_rec<R, N>(x, p);
  }
}

template <typename R, int N>
__device__ __forceinline__ void store_rec(void* p, const Cx<R> (&x)[N]) {
  if constexpr (sizeof(R) == 4) {
    float2* q = reinterpret_cast<float2*>(p);
#pragma unroll
    for (int e = 0; e < N; e++) q[e] = make_float2(x[e].re, x[e].im);
  } else {
    double2* q = reinterpret_cast<double2*>(p);
#pragma unroll
    for (int e = 0; e < N; e++) q[e] = make_double2(x[e].re, x[e].im);
  }
}

// ---------------------------------------------------------------------------
// sm_90+/sm_100a asynchronous-copy primitives (inline PTX).
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Time-bounded wait on an mbarrier phase: gives up after ~limit_ns (or at
// once when *abort becomes non-zero) and records QLA_DEVERR_MBAR_TIMEOUT.
// Returns false on timeout / abort.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, unsigned* err,
                                                  uint64_t limit_ns = 2000000000ull,
                                                  volatile int* abort = nullptr) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0; it < (1u << 30); ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 15u) == 0) {
      if (abort && *abort) return false;
      if (global_ns() - t0 > limit_ns) break;
    }
  }
  raise_dev_error(err, QLA_DEVERR_MBAR_TIMEOUT);
  return false;
}

// The same wait for a thread with nothing else to do (a producer lane ahead
// of its consumers, a consumer ahead of its data): each try suspends the
// thread for up to hint_ns or until the phase completes, so that waiting
// warps do not take issue slots from the computing ones.
__device__ __forceinline__ bool mbar_try_wait_hint(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded_idle(uint64_t* bar, uint32_t parity, unsigned* err,
                                                       uint64_t limit_ns = 2000000000ull,
                                                       volatile int* abort = nullptr, uint32_t hint_ns = 20000u) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0; it < (1u << 30); ++it) {
    if (mbar_try_wait_hint(bar, parity, hint_ns)) return true;
    if (abort && *abort) return false;
    if (global_ns() - t0 > limit_ns) break;
  }
  raise_dev_error(err, QLA_DEVERR_MBAR_TIMEOUT);
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// A consumer warp hands a staged tile back to the producer.  The warp's
// shared-memory reads of the stage (generic proxy) must be complete before
// the producer's next bulk copy (async proxy) lands in it.  The mbarrier
// arrive by itself did not ensure that on B200: a D3 norm2 of 192-B records
// read stage data that the next tile's copy had already overwritten.  After
// the warp has converged, the arriving lane issues a generic-to-async proxy
// fence first; the loads are warp-wide instructions, so that lane's fence
// covers every lane's reads.  (A full block-scope memory fence in every lane
// also works but costs 14% on the axpy kernel; this costs ~2%.)
__device__ __forceinline__ void release_stage(uint64_t* bar, int lane) {
  __syncwarp();
  if (lane == 0) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_arrive(bar);
  }
}

// 1-D bulk copy global -> shared, completion signalled on an mbarrier.
// Requires 16-B aligned addresses and a size that is a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar,
                                        uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], "
      "%4;" ::"r"(smem_addr(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}

// 1-D bulk copy shared -> global, tracked by the issuing thread's bulk groups.
__device__ __forceinline__ void bulk_s2g(void* dst_gmem, const void* src_smem, uint32_t bytes, uint64_t policy) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group.L2::cache_hint [%0], [%1], %2, %3;" ::"l"(dst_gmem),
               "r"(smem_addr(src_smem)), "r"(bytes), "l"(policy)
               : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

template <int N>
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Prefetch the L2 line holding a global address (no register result).
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// L2 eviction policies for streamed data (read once / written once).
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_normal() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// ---------------------------------------------------------------------------
// double-double accumulation (Knuth TwoSum) for the global reductions.
struct DD {
  double hi, lo;
};

__device__ __forceinline__ void dd_add(DD& s, double x) {
  double t = __dadd_rn(s.hi, x);
  double bp = __dsub_rn(t, s.hi);
  double err = __dadd_rn(__dsub_rn(s.hi, __dsub_rn(t, bp)), __dsub_rn(x, bp));
  s.hi = t;
  s.lo = __dadd_rn(s.lo, err);
}

__device__ __forceinline__ void dd_merge(DD& s, const DD& o) {
  dd_add(s, o.hi);
  s.lo = __dadd_rn(s.lo, o.lo);
}

// sum of U doubles (U a power of two) by a fixed pairwise tree: at most U - 1
// roundings, each within half an ulp of the group's magnitude.  Reductions
// sum each thread's group of in-flight terms this way and add the group sum
// in double-double, so one accumulator serves U loads in flight.
template <int U>
__device__ __forceinline__ double tree_sum(const double (&v)[U]) {
  static_assert((U & (U - 1)) == 0, "tree_sum needs a power of two");
  double w[U];
#pragma unroll
  for (int u = 0; u < U; u++) w[u] = v[u];
#pragma unroll
  for (int h = U / 2; h >= 1; h >>= 1)
#pragma unroll
    for (int u = 0; u < h; u++) w[u] = __dadd_rn(w[u], w[u + h]);
  return w[0];
}

__device__ __forceinline__ DD dd_shfl_xor(const DD& v, int lane_mask) {
  DD o;
  o.hi = __shfl_xor_sync(0xffffffffu, v.hi, lane_mask);
  o.lo = __shfl_xor_sync(0xffffffffu, v.lo, lane_mask);
  return o;
}

}  // namespace qlab
