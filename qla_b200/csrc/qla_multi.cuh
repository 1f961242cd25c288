// qla_multi.cuh -- multi-direction accumulation
//     r[i] (eqop) sum_d A_d[i] * b_d[i],   d = 0 .. nd-1
// (QLA_F3/D3 V_{v,x}{eqop}_n{p}M{a}_times_n{p}V, build_qla.pl:1693-1727; the
// hand-optimised lib/optimized/c/src/QLA_D3_V_vpeq_nM_times_npV.c is the same
// operation).  The reference rounds r after every direction: direction 0
// starts from 0 (eq, eqm) or r (peq, meq), every later direction from the
// rounded r, with the eqop's sign; the kernel keeps that order, so the result
// is bit-identical, but reads and writes r once instead of nd times.
//
// The operand arrays a, b (nd pointers to fields, or to per-site pointer
// arrays for the `np` forms) may be host or device memory; their entries are
// passed to the kernel by value, up to kMaxDirs per launch (larger nd run in
// consecutive launches, which gives the same rounding sequence).
#pragma once
#include "qla_launch.cuh"
#include "qla_ops.cuh"

namespace qlab {

constexpr int kMaxDirs = 8;

struct MultiParams {
  Opnd a[kMaxDirs], b[kMaxDirs];
  void* out;
  const int* gang;
  long long n;
  int nd;
  int eqop;       // eqop of direction 0 of this launch
  int minus;      // sign of every direction
  int out_read;   // direction 0 starts from r
  unsigned stage_bytes, tx_bytes;
  unsigned off_a[kMaxDirs], off_b[kMaxDirs], off_r;
  int stages;
  long long ntiles;
  unsigned* err;
};

template <typename R, bool ADJ>
__device__ __forceinline__ void multi_site(const MultiParams& p, const Cx<R> (&a)[9], const Cx<R> (&b)[3],
                                           Cx<R> (&y)[3], bool load) {
  lmult_site<R, 3, 1, ADJ, false>(p.minus ? MEQ : PEQ, load, a, b, y);
}

// direct path (gang index, unaligned pointers, partial tiles): one site
template <typename R, bool ADJ>
__device__ __forceinline__ void multi_site_direct(const MultiParams& p, long long k) {
  constexpr int OB = 3 * (int)sizeof(Cx<R>);
  char* dst = static_cast<char*>(p.out) + k * OB;
  Cx<R> y[3];
  if (p.out_read) load_rec_rw<R, 3>(y, dst);
  for (int d = 0; d < p.nd; d++) {
    Cx<R> a[9], b[3];
    fetch_gathered<LMultOp<R, 3, 1, ADJ, false>, 9>(a, p.a[d], k);
    fetch_gathered<LMultOp<R, 3, 1, ADJ, false>, 3>(b, p.b[d], k);
    multi_site<R, ADJ>(p, a, b, y, d > 0 || p.out_read);
  }
  store_rec<R, 3>(dst, y);
}

template <typename R, bool ADJ>
__global__ void __launch_bounds__(256) multi_direct_kernel(const MultiParams p) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += stride)
    multi_site_direct<R, ADJ>(p, p.gang ? (long long)p.gang[i] : i);
}

// warp-specialised bulk-copy pipeline, as site_tma_kernel, with 2*nd (+1)
// operand tiles per stage
template <typename R, bool ADJ>
__global__ void __launch_bounds__(288) multi_tma_kernel(const MultiParams p) {
  constexpr int RM = 9 * (int)sizeof(Cx<R>), RV = 3 * (int)sizeof(Cx<R>);
  extern __shared__ __align__(128) unsigned char smem[];
  const int S = p.stages;
  const int NW = (blockDim.x >> 5) - 1;
  const int T = NW * 32;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + 8;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + 128);
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
  bool alive = true;
  long long issued = 0;
  if (warp == NW) {
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
        const long long site0 = ((long long)blockIdx.x + k * gridDim.x) * T;
        unsigned char* st = stages + (size_t)s * p.stage_bytes;
        mbar_arrive_expect_tx(&full[s], p.tx_bytes);
        for (int d = 0; d < p.nd; d++) {
          const Opnd& oa = p.a[d];
          const Opnd& ob = p.b[d];
          if (oa.mode == OM_CONTIG)
            bulk_g2s(st + p.off_a[d], static_cast<const char*>(oa.base) + site0 * RM, (unsigned)T * RM, &full[s], pol);
          else
            bulk_g2s(st + p.off_a[d], oa.ptrs + site0, (unsigned)T * 8u, &full[s], pol);
          if (ob.mode == OM_CONTIG)
            bulk_g2s(st + p.off_b[d], static_cast<const char*>(ob.base) + site0 * RV, (unsigned)T * RV, &full[s], pol);
          else
            bulk_g2s(st + p.off_b[d], ob.ptrs + site0, (unsigned)T * 8u, &full[s], pol);
        }
        if (p.out_read)
          bulk_g2s(st + p.off_r, static_cast<const char*>(p.out) + site0 * RV, (unsigned)T * RV, &full[s], pol);
        if (++s == S) {
          s = 0;
          round++;
        }
      }
      issued = k;
    }
  } else {
    const uint64_t pol = policy_evict_first();
    unsigned char* myout = outbuf + (size_t)warp * 2 * 32 * RV;
    int s = 0;
    uint32_t par = 0;
    const int t = warp * 32 + lane;
    for (long long k = 0; k < my; k++) {
      if (!mbar_wait_bounded(&full[s], par, p.err, 2000000000ull, abort_flag)) {
        *abort_flag = 1;
        alive = false;
        break;
      }
      const unsigned char* st = stages + (size_t)s * p.stage_bytes;
      Cx<R> y[3];
      if (p.out_read) load_rec<R, 3>(y, st + p.off_r + (unsigned)t * RV);
      for (int d = 0; d < p.nd; d++) {
        Cx<R> a[9], b[3];
        fetch_staged<LMultOp<R, 3, 1, ADJ, false>, 9>(a, p.a[d], st, p.off_a[d], t);
        fetch_staged<LMultOp<R, 3, 1, ADJ, false>, 3>(b, p.b[d], st, p.off_b[d], t);
        multi_site<R, ADJ>(p, a, b, y, d > 0 || p.out_read);
      }
      unsigned char* ob = myout + (size_t)(k & 1) * 32 * RV;
      if (lane == 0) bulk_wait_read<1>();
      __syncwarp();
      store_rec_smem<R, 3>(ob + (unsigned)lane * RV, y);
      // orders this lane's stage reads and slice writes before the async
      // proxy (the store below and the producer's next copy into the stage)
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&empty[s]);  // this warp is done with the stage
        const long long site0 = ((long long)blockIdx.x + k * gridDim.x) * T + warp * 32;
        bulk_s2g(static_cast<char*>(p.out) + site0 * RV, ob, 32u * RV, pol);
        bulk_commit();
      }
      if (++s == S) {
        s = 0;
        par ^= 1u;
      }
    }
    if (lane == 0) bulk_wait_all<0>();
    if (alive && blockIdx.x == gridDim.x - 1) {
      const long long k0 = p.ntiles * T + t;
      if (k0 < p.n) multi_site_direct<R, ADJ>(p, k0);
    }
  }
  __syncthreads();
  if (*abort_flag && warp == NW && lane == 0) {
    for (long long kk = (issued > S ? issued - S : 0); kk < issued; kk++)
      if (!mbar_wait_bounded(&full[kk % S], (uint32_t)((kk / S) & 1), p.err, 200000000ull, nullptr))
        raise_dev_error(p.err, QLA_DEVERR_BULK_TIMEOUT);
  }
}

// fetch the nd operand entries (host or device array) into ops[]
inline bool multi_fetch_ptrs(const void* arr, int nd, const void** out) {
  if (is_device_ptr(arr)) {
    if (cudaMemcpy(out, arr, sizeof(void*) * (size_t)nd, cudaMemcpyDeviceToHost) != cudaSuccess) return false;
  } else {
    std::memcpy(out, arr, sizeof(void*) * (size_t)nd);
  }
  return true;
}

// r (eqop) sum_d A_d * b_d.  pa / pb: the operands are per-site pointer arrays.
template <typename R, bool ADJ>
inline void api_multi(const char* kid, void* r, const void* a, bool pa, const void* b, bool pb, const int* gang,
                      int n, int nd, int eqop) {
  if (n <= 0 || nd <= 0) return;  // the reference's loops run zero times
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
  constexpr int RM = 9 * (int)sizeof(Cx<R>), RV = 3 * (int)sizeof(Cx<R>);
  cudaStream_t st = current_stream();
  const int sms = device_sm_count();
  for (int d0 = 0; d0 < nd; d0 += kMaxDirs) {
    MultiParams p;
    std::memset(&p, 0, sizeof(p));
    p.nd = (nd - d0 < kMaxDirs) ? nd - d0 : kMaxDirs;
    p.out = r;
    p.gang = gang;
    p.n = n;
    p.minus = (eqop == MEQ || eqop == EQM) ? 1 : 0;
    // later chunks continue the accumulation from the rounded r
    p.out_read = (d0 > 0 || eqop == PEQ || eqop == MEQ) ? 1 : 0;
    p.eqop = eqop;
    p.err = device_error_word();
    bool direct = (gang != nullptr) || !aligned16(r);
    for (int d = 0; d < p.nd; d++) {
      const void* ad = av[(size_t)(d0 + d)];
      const void* bd = bv[(size_t)(d0 + d)];
      p.a[d] = pa ? op_ptr(static_cast<const void* const*>(ad)) : op_contig(ad);
      p.b[d] = pb ? op_ptr(static_cast<const void* const*>(bd)) : op_contig(bd);
      direct = direct || !aligned16(ad) || !aligned16(bd);
    }
    // pointer (gathered) operands whose staged bytes per site leave tiles of
    // fewer than 128 sites run the direct kernel: with few sites staged per
    // block the gathers' latency is exposed.  Measured on B200, D3
    // V_vpeq_nM_times_npV at nd = 4 (656 B staged per site, 64-site tiles),
    // 32^3 x 64 sites: staged 345 us, direct 264 us; F3 (344 B, 128-site
    // tiles) stays staged at 0.98 of HBM peak.
    const unsigned staged_bps = (unsigned)p.nd * ((pa ? 8u : RM) + (pb ? 8u : RV)) + (p.out_read ? RV : 0u);
    if ((pa || pb) && default_shape(staged_bps, RV).threads < 128) direct = true;
    if (direct) {
      long long grid = ((long long)n + 255) / 256;
      if (grid > (long long)sms * 8) grid = (long long)sms * 8;
      multi_direct_kernel<R, ADJ><<<(unsigned)(grid < 1 ? 1 : grid), 256, 0, st>>>(p);
    } else {
      const unsigned bps = (unsigned)p.nd * ((pa ? 8u : RM) + (pb ? 8u : RV)) + (p.out_read ? RV : 0u);
      LaunchShape sh = default_shape(bps, RV);
      while (tma_smem_bytes(sh.threads, sh.stages, stage_bytes_for(sh.threads, bps), RV) > 225u * 1024u &&
             sh.threads > 32)
        sh.threads /= 2;
      const int T = sh.threads;
      unsigned off = 0;
      for (int d = 0; d < p.nd; d++) {
        p.off_a[d] = off;
        off += (unsigned)T * (pa ? 8u : RM);
        p.off_b[d] = off;
        off += (unsigned)T * (pb ? 8u : RV);
      }
      p.off_r = off;
      if (p.out_read) off += (unsigned)T * RV;
      p.tx_bytes = off;
      p.stage_bytes = (off + 127u) & ~127u;
      p.stages = sh.stages;
      p.ntiles = (long long)n / T;
      const size_t smem = tma_smem_bytes(T, p.stages, p.stage_bytes, RV);
      const void* fn = reinterpret_cast<const void*>(&multi_tma_kernel<R, ADJ>);
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      int nb = 1;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, T + 32, smem) != cudaSuccess || nb < 1) nb = 1;
      long long grid = (long long)nb * sms;
      if (grid > p.ntiles) grid = p.ntiles;
      if (grid < 1) grid = 1;
      void* args[] = {&p};
      if (cudaLaunchKernel(fn, dim3((unsigned)grid), dim3((unsigned)T + 32u), args, smem, st) != cudaSuccess) {
        check_launch(kid);
        return;
      }
    }
    if (!check_launch(kid)) return;
  }
}

}  // namespace qlab
