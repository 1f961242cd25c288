// qla_launch.cuh -- host-side launch of an engine OP: path selection (bulk-copy
// pipeline vs direct), tile shape, occupancy-sized persistent grid, reduction
// scratch and the synchronous host-result semantics of the reference.
#pragma once
#include <cstring>
#include <mutex>
#include <map>
#include <tuple>

#include "qla_engine.cuh"
#include "qla_runtime.h"

namespace qlab {

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

struct LaunchShape {
  int threads;  // sites per tile == threads per block
  int stages;
};

// shared memory of one block of the pipelined kernel
inline size_t tma_smem_bytes(int threads, int stages, unsigned stage_bytes, unsigned out_bytes) {
  return 256 + (size_t)stages * stage_bytes + 2 * (size_t)threads * out_bytes;
}

inline unsigned stage_bytes_for(int threads, unsigned bytes_per_site) {
  return ((unsigned)threads * bytes_per_site + 127u) & ~127u;
}

// Default tile shape: two stages, and the largest tile (sites = consumer
// threads) whose block still fits in ~100 KB of shared memory, so that two to
// four blocks share an SM.  Measured on B200: more resident blocks beat deeper
// pipelines for these streaming tiles.
inline LaunchShape default_shape(unsigned bytes_per_site, unsigned out_bytes) {
  LaunchShape s{64, 2};
  for (int t : {256, 128, 64}) {
    if (tma_smem_bytes(t, 2, stage_bytes_for(t, bytes_per_site), out_bytes) <= 100u * 1024u) {
      s.threads = t;
      break;
    }
  }
  return s;
}

template <class OP>
struct SiteLauncher {
  using R = typename OP::R;
  static constexpr int RB[3] = {OP::N0 * (int)sizeof(Cx<R>), OP::N1 * (int)sizeof(Cx<R>),
                                OP::N2 * (int)sizeof(Cx<R>)};
  static constexpr int OB = OP::NOUT * (int)sizeof(Cx<R>);

  static int blocks_per_sm(const void* fn, int threads, size_t smem) {
    static std::mutex mu;
    static std::map<std::tuple<int, int, size_t, const void*>, int> cache;
    const int dev = current_device();
    auto key = std::make_tuple(dev, threads, smem, fn);
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, smem) != cudaSuccess) nb = 1;
    if (nb < 1) nb = 1;
    cache[key] = nb;
    return nb;
  }

  static void set_smem_attr(const void* fn, size_t smem) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> done;
    const int dev = current_device();
    std::lock_guard<std::mutex> g(mu);
    size_t& cur = done[std::make_pair(dev, fn)];
    if (smem > cur) {
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      cur = smem;
    }
  }

  // kernel_id names the OP for the autotuner table
  static void run(SiteParams p, const char* kernel_id, void* host_result = nullptr, size_t result_bytes = 0) {
    constexpr bool reduce = OP::NACC > 0;
    cudaStream_t st = current_stream();
    if (p.n <= 0) {
      // the reference loops zero times; reductions still store their (zero) sum
      if (reduce) {
        if (host_result)
          std::memset(host_result, 0, result_bytes);
        else if (p.result)
          cudaMemsetAsync(p.result, 0, result_bytes, st);
      }
      return;
    }
    p.err = device_error_word();
    // ---- path selection
    bool direct = (p.gang != nullptr);
    for (int j = 0; j < OP::NIN; j++) {
      const Opnd& o = p.in[j];
      const void* q = o.mode == OM_PTR ? (const void*)o.ptrs : (o.mode == OM_IDX ? (const void*)o.idx : o.base);
      if (!aligned16(q)) direct = true;
    }
    if (OP::NOUT > 0 && !aligned16(p.out)) direct = true;

    // ---- reduction scratch / result destination
    ReduceScratch* rs = nullptr;
    int sms = device_sm_count();
    if (reduce) {
      rs = reduce_scratch(st, 32 * sms + 64);
      if (!rs) return;
      p.partials = rs->partials;
      p.counter = rs->counter;
      if (host_result) p.result = rs->result;
    }

    if (direct) {
      const int threads = 256;
      long long want = (p.n + threads - 1) / threads;
      long long cap = (long long)sms * 8;
      int grid = (int)(want < cap ? want : cap);
      if (grid < 1) grid = 1;
      site_direct_kernel<OP><<<grid, threads, 0, st>>>(p);
    } else {
      unsigned bps = 0;
      for (int j = 0; j < OP::NIN; j++)
        bps += p.in[j].mode == OM_CONTIG ? RB[j] : (p.in[j].mode == OM_PTR ? 8u : 4u);
      if (OP::NOUT > 0 && p.out_read) bps += OB;
      LaunchShape sh = default_shape(bps, OB);
      int tt, ts;
      char key[96];
      {
        int q = 0;
        for (const char* c = kernel_id; *c && q < 80; c++) key[q++] = *c;
        key[q++] = ':';
        for (int j = 0; j < OP::NIN; j++) key[q++] = "-cpi"[p.in[j].mode & 3];
        if (OP::NOUT > 0 && p.out_read) key[q++] = 'r';
        key[q] = 0;
      }
      if (tuned_shape(key, &tt, &ts)) {
        sh.threads = tt;
        sh.stages = ts;
      }
      // stay within the per-block shared-memory limit (227 KB less the static
      // reduction scratch): shed stages, then halve the tile down to one warp,
      // then (very large records, e.g. nc = 8 matrices) run unpipelined
      while (tma_smem_bytes(sh.threads, sh.stages, stage_bytes_for(sh.threads, bps), OB) > 225u * 1024u) {
        if (sh.stages > 2)
          sh.stages--;
        else if (sh.threads > 32)
          sh.threads /= 2;
        else if (sh.stages > 1)
          sh.stages = 1;
        else
          break;
      }
      const int T = sh.threads;
      unsigned off = 0;
      p.tx_bytes = 0;
      for (int j = 0; j < OP::NIN; j++) {
        p.off_in[j] = off;
        unsigned b = (unsigned)T * (p.in[j].mode == OM_CONTIG ? RB[j] : (p.in[j].mode == OM_PTR ? 8u : 4u));
        off += (b + 15u) & ~15u;
        p.tx_bytes += b;
      }
      p.off_out_in = off;
      if (OP::NOUT > 0 && p.out_read) {
        off += (unsigned)T * OB;
        p.tx_bytes += (unsigned)T * OB;
      }
      p.stage_bytes = (off + 127u) & ~127u;
      p.ntiles = p.n / T;
      p.stages = sh.stages;
      const size_t smem = tma_smem_bytes(T, p.stages, p.stage_bytes, OB);
      const void* fn = reinterpret_cast<const void*>(&site_tma_kernel<OP>);
      set_smem_attr(fn, smem);
      const int nb = blocks_per_sm(fn, T + 32, smem);
      long long grid = (long long)nb * sms;
      if (grid > p.ntiles) grid = p.ntiles;
      if (grid < 1) grid = 1;
      if (reduce && grid > rs->max_blocks) grid = rs->max_blocks;
      void* args[] = {&p};
      // T consumer threads + one producer warp
      if (cudaLaunchKernel(fn, dim3((unsigned)grid), dim3((unsigned)T + 32u), args, smem, st) != cudaSuccess) {
        check_launch(kernel_id);
        return;
      }
    }
    if (!check_launch(kernel_id)) return;
    if (reduce && host_result) {
      if (cudaMemcpyAsync(host_result, rs->result, result_bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess)
        check_launch(kernel_id);
    }
  }
};

// operand constructors
inline Opnd op_contig(const void* base) { return Opnd{base, nullptr, nullptr, OM_CONTIG}; }
inline Opnd op_ptr(const void* const* ptrs) { return Opnd{nullptr, ptrs, nullptr, OM_PTR}; }
inline Opnd op_idx(const void* base, const int* idx) { return Opnd{base, nullptr, idx, OM_IDX}; }

inline SiteParams make_params(long long n, int eqop) {
  SiteParams p;
  std::memset(&p, 0, sizeof(p));
  p.n = n;
  p.eqop = eqop;
  p.out_read = (eqop == PEQ || eqop == MEQ) ? 1 : 0;
  return p;
}

}  // namespace qlab
