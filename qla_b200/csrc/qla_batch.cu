// qla_batch.cu -- many fields of uneven volume in one persistent launch.
//
// A lattice code often applies the same short level-1 sequence to many
// independent fields (sub-lattices, sources, time slices).  Launching QLA's
// functions once per field costs a launch each and leaves the GPU idle on
// the small fields.  Here a plan flattens the fields' tiles into one global
// tile list (prefix sums over per-field tile counts, kept on the device) and
// one persistent, warp-specialised bulk-copy pipeline walks that list.
//
// The sequence is, per field f and site i:
//     r_f[i] = u_f[i] * u2_f[nbr_f[i]]      (QLA_F3_M_eq_M_times_xM, int32 neighbour gather)
//     w_f[i] = r_f[i] * v_f[i]              (QLA_F3_V_veq_M_times_V)
// Both are site-local, so one block computes both for a tile without any
// dependency on other blocks; r is kept in registers between the two and
// still written out.  Results are bit-identical to the two separate calls.
//
// The launch itself (qlagpu_batch_run) only passes the plan's device pointer:
// it can be replayed from a captured CUDA graph.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "../../include/qla_b200_runtime.h"
#include "qla_launch.cuh"
#include "qla_ops.cuh"

namespace qlab {

struct BatchField {
  float* r;
  const float* u;
  const float* u2;
  const int* nbr;
  float* w;
  const float* v;
  long long n;
  long long tile0;  // first global tile of this field
  int direct;       // 1: pointers not 16-B aligned, every tile by plain loads
  int pad;
};

struct BatchPlan {
  BatchField* dfields;  // device copy
  int nfields;
  long long ntiles;
  int threads;  // consumer threads = sites per tile
  int stages;
  int device;
  int grid;
  size_t smem;
};

struct BatchParams {
  const BatchField* fields;
  int nfields;
  long long ntiles;
  int stages;
  unsigned stage_bytes;
  unsigned* err;
};

using MxM = LMultOp<float, 3, 3, false, false>;
using MxV = LMultOp<float, 3, 1, false, false>;
constexpr int kRecM = 72, kRecV = 24;

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

// one site, plain loads/stores (partial tiles and unaligned fields)
__device__ __forceinline__ void batch_site_direct(const BatchField& F, long long i, const SiteParams& sp) {
  Cx<float> u[9], g[9], v[3], r[9], w[3];
  Cx<float> dummy[1];
  load_rec_global<float, 9>(u, F.u + i * 18);
  load_rec_global<float, 9>(g, F.u2 + (long long)F.nbr[i] * 18);
  load_rec_global<float, 3>(v, F.v + i * 6);
  MxM::apply(sp, u, g, dummy, r);
  MxV::apply(sp, r, v, dummy, w);
  store_rec<float, 9>(F.r + i * 18, r);
  store_rec<float, 3>(F.w + i * 6, w);
}

// Dynamic smem: [full[8], empty[8], abort, field table | S stages (U, idx, V)
//               | NW x 2 slices of 32 (R, W) records]
__global__ void __launch_bounds__(288) batch_mxm_mxv_kernel(const BatchParams p) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int S = p.stages;
  const int NW = (blockDim.x >> 5) - 1;
  const int T = NW * 32;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + 8;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + 128);
  long long* tile0 = reinterpret_cast<long long*>(smem + 256);  // up to 1024 fields
  unsigned char* stages = smem + 256 + 8 * 1024;
  unsigned char* outbuf = stages + (size_t)S * p.stage_bytes;
  const unsigned offI = (unsigned)T * kRecM, offV = offI + (unsigned)T * 4;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long my =
      ((long long)blockIdx.x < p.ntiles) ? (p.ntiles - 1 - (long long)blockIdx.x) / gridDim.x + 1 : 0;

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

  SiteParams sp;  // the per-site ops only read eqop / out_read
  sp.eqop = EQ;
  sp.out_read = 0;
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
        const long long g = (long long)blockIdx.x + k * gridDim.x;
        const BatchField& F = p.fields[find_field(tile0, p.nfields, g)];
        const long long site0 = (g - F.tile0) * T;
        unsigned char* st = stages + (size_t)s * p.stage_bytes;
        if (!F.direct && site0 + T <= F.n) {
          mbar_arrive_expect_tx(&full[s], (unsigned)T * (kRecM + 4 + kRecV));
          bulk_g2s(st, F.u + site0 * 18, (unsigned)T * kRecM, &full[s], pol);
          bulk_g2s(st + offI, F.nbr + site0, (unsigned)T * 4, &full[s], pol);
          bulk_g2s(st + offV, F.v + site0 * 6, (unsigned)T * kRecV, &full[s], pol);
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
    const uint64_t pol = policy_evict_first();
    unsigned char* myout = outbuf + (size_t)warp * 2 * 32 * (kRecM + kRecV);
    int s = 0;
    uint32_t par = 0;
    for (long long k = 0; k < my; k++) {
      if (!mbar_wait_bounded(&full[s], par, p.err, 2000000000ull, abort_flag)) {
        *abort_flag = 1;
        break;
      }
      const long long g = (long long)blockIdx.x + k * gridDim.x;
      const BatchField& F = p.fields[find_field(tile0, p.nfields, g)];
      const long long site0 = (g - F.tile0) * T;
      const int t = warp * 32 + lane;
      if (!F.direct && site0 + T <= F.n) {
        const unsigned char* st = stages + (size_t)s * p.stage_bytes;
        Cx<float> u[9], gm[9], v[3], r[9], w[3], dummy[1];
        load_rec<float, 9>(u, st + (unsigned)t * kRecM);
        const int j = reinterpret_cast<const int*>(st + offI)[t];
        load_rec<float, 3>(v, st + offV + (unsigned)t * kRecV);
        load_rec_global<float, 9>(gm, F.u2 + (long long)j * 18);
        MxM::apply(sp, u, gm, dummy, r);
        MxV::apply(sp, r, v, dummy, w);
        unsigned char* ob = myout + (size_t)(k & 1) * 32 * (kRecM + kRecV);
        if (lane == 0) bulk_wait_read<1>();
        __syncwarp();
        store_rec_smem<float, 9>(ob + (unsigned)lane * kRecM, r);
        store_rec_smem<float, 3>(ob + 32 * kRecM + (unsigned)lane * kRecV, w);
        // orders this lane's stage reads and slice writes before the async
        // proxy (the stores below and the producer's next copy into the stage)
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&empty[s]);  // this warp is done with the stage
          const long long s0 = site0 + warp * 32;
          bulk_s2g(F.r + s0 * 18, ob, 32u * kRecM, pol);
          bulk_s2g(F.w + s0 * 6, ob + 32 * kRecM, 32u * kRecV, pol);
          bulk_commit();
        }
      } else {
        release_stage(&empty[s], lane);  // this warp is done with the stage
        const long long i = site0 + t;
        if (i < F.n) batch_site_direct(F, i, sp);
        if (lane == 0) bulk_commit();  // an empty group keeps the slice bookkeeping aligned
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
    for (long long kk = (issued > S ? issued - S : 0); kk < issued; kk++)
      if (!mbar_wait_bounded(&full[kk % S], (uint32_t)((kk / S) & 1), p.err, 200000000ull, nullptr))
        raise_dev_error(p.err, QLA_DEVERR_BULK_TIMEOUT);
  }
}

}  // namespace qlab

using namespace qlab;

extern "C" QLAB_EXPORT void* qlagpu_F3_batch_plan(const qlagpu_F3_batch_field* fields, int nfields) {
  const char* who = "qlagpu_F3_batch_plan";
  if (!fields || nfields <= 0 || nfields > 1024) {
    set_error(QLAGPU_ERR_ARG, who, "need 1 <= nfields <= 1024 and a field table");
    return nullptr;
  }
  int t = 128, st = 3;
  if (!tuned_shape("F3_batch_mxm_mxv", &t, &st)) {
    t = 128;
    st = 3;
  }
  std::vector<BatchField> h((size_t)nfields);
  long long tiles = 0;
  for (int f = 0; f < nfields; f++) {
    const qlagpu_F3_batch_field& q = fields[f];
    if (!q.r || !q.u || !q.u2 || !q.nbr || !q.w || !q.v || q.n < 0) {
      set_error(QLAGPU_ERR_NULLPTR, who, "NULL array in a field (or n < 0)");
      return nullptr;
    }
    BatchField& b = h[(size_t)f];
    b.r = reinterpret_cast<float*>(q.r);
    b.u = reinterpret_cast<const float*>(q.u);
    b.u2 = reinterpret_cast<const float*>(q.u2);
    b.nbr = q.nbr;
    b.w = reinterpret_cast<float*>(q.w);
    b.v = reinterpret_cast<const float*>(q.v);
    b.n = q.n;
    b.tile0 = tiles;
    b.direct = !(aligned16(q.r) && aligned16(q.u) && aligned16(q.nbr) && aligned16(q.w) && aligned16(q.v));
    b.pad = 0;
    tiles += (q.n + t - 1) / t;
  }
  if (!device_error_word()) return nullptr;  // allocate it now, not inside a later capture
  BatchPlan* plan = new BatchPlan();
  plan->nfields = nfields;
  plan->ntiles = tiles;
  plan->threads = t;
  plan->stages = st;
  plan->device = current_device();
  if (cudaMalloc(&plan->dfields, sizeof(BatchField) * (size_t)nfields) != cudaSuccess ||
      cudaMemcpy(plan->dfields, h.data(), sizeof(BatchField) * (size_t)nfields, cudaMemcpyHostToDevice) !=
          cudaSuccess) {
    check_launch(who);
    set_error(QLAGPU_ERR_ALLOC, who, "plan table allocation failed");
    delete plan;
    return nullptr;
  }
  const unsigned stage_bytes = ((unsigned)t * (kRecM + 4 + kRecV) + 127u) & ~127u;
  plan->smem = 256 + 8 * 1024 + (size_t)st * stage_bytes + 2 * (size_t)t * (kRecM + kRecV);
  const void* fn = reinterpret_cast<const void*>(&batch_mxm_mxv_kernel);
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plan->smem);
  int nb = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, t + 32, plan->smem) != cudaSuccess || nb < 1) nb = 1;
  long long grid = (long long)nb * device_sm_count();
  if (grid > tiles) grid = tiles;
  plan->grid = (int)(grid < 1 ? 1 : grid);
  return plan;
}

extern "C" QLAB_EXPORT int qlagpu_batch_run(void* handle) {
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
  p.stage_bytes = ((unsigned)plan->threads * (kRecM + 4 + kRecV) + 127u) & ~127u;
  p.err = device_error_word();
  void* args[] = {&p};
  if (cudaLaunchKernel(reinterpret_cast<const void*>(&batch_mxm_mxv_kernel), dim3((unsigned)plan->grid),
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
