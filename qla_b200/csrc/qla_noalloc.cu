// qla_noalloc.cu -- a global norm2 of a DiracFermion field that allocates no
// device memory at all.
//
// Who needs it: some host programs cannot call cudaMalloc while they run.  A
// lattice code whose own pool allocator reserved the device memory up front
// may find nothing left for a library to allocate, or must not let a library
// fragment its pool; code working under a hard memory budget cannot risk an
// allocation failing in the middle of a solve.  The regular reduction entry
// points allocate their scratch (per-block partial sums and a ticket counter)
// lazily on first use, so such callers get this variant instead.
//
// Scratch lives in one file-scope static device array of a fixed size: every
// GPU that loads the library holds it until the process exits.  Its device
// address is obtained once per device with cudaGetSymbolAddress (host code
// may not use the array's name as an address: on the host that name only
// stands in for the device symbol).
//
// Shape: one 256-site tile per block (the pipelined kernel of the regular
// entry points, with a grid of one block per tile), so the scratch holds one
// partial per tile and bounds the field size: at most
// kMaxPartials * kSitesPerTile = 16,777,216 sites; larger n are rejected.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/qla_b200_runtime.h"
#include "../../include/qla_b200_types.h"
#include "qla_launch.cuh"
#include "qla_ops.cuh"

namespace qlab {
namespace noalloc {

constexpr int kSitesPerTile = 256;
constexpr int kStages = 2;
constexpr int kMaxPartials = 65536;
constexpr long long kMaxSites = (long long)kMaxPartials * kSitesPerTile;
// layout: [partials: kMaxPartials DD][result: 2 doubles][counter][per-call
// error word][sticky error word]
constexpr size_t kOffResult = sizeof(DD) * (size_t)kMaxPartials;
constexpr size_t kOffCounter = kOffResult + 2 * sizeof(double);
constexpr size_t kOffErr = kOffCounter + sizeof(unsigned);
constexpr size_t kOffSticky = kOffErr + sizeof(unsigned);
constexpr size_t kScratchBytes = kOffErr + 256;  // 1 MiB + 272 B

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

using Op = Norm2Op<float, 12, double>;  // QLA_DF3_r_veq_norm2_D

constexpr unsigned kRecBytes = Op::N0 * sizeof(Cx<float>);
inline unsigned tile_stage_bytes() { return stage_bytes_for(kSitesPerTile, kRecBytes); }
inline size_t tile_smem_bytes() { return tma_smem_bytes(kSitesPerTile, kStages, tile_stage_bytes(), 0); }

// Once per device, with that device current (the first call on a device does
// this set-up): the device address of the scratch, and the pipelined
// kernel's shared-memory limit raised to what this file's tile needs.  The
// limit is a property of the kernel shared with the regular norm2 entry
// point, so it goes through the launcher's helper, which only ever raises it.
static unsigned char* scratch_on_current_device() {
  static std::mutex mu;
  static unsigned char* addr[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return nullptr;
  }
  std::lock_guard<std::mutex> g(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return nullptr;
    }
    SiteLauncher<Op>::set_smem_attr(reinterpret_cast<const void*>(&site_tma_kernel<Op>), tile_smem_bytes());
    if (cudaGetLastError() != cudaSuccess) return nullptr;
    addr[dev] = static_cast<unsigned char*>(p);
  }
  return addr[dev];
}

// After the reduction: the call's error bits go into the sticky word (read and
// cleared by qlagpu_device_error), and a device result is overwritten with a
// NaN when a wait gave up, so that a caller who never asks still cannot take
// an incomplete sum for a valid one.
__global__ void noalloc_fold_error(const unsigned* err, unsigned* sticky, double* dev_result) {
  const unsigned e = *err;
  if (e) {
    atomicOr(sticky, e);
    if (dev_result) *dev_result = __longlong_as_double(0x7ff8000000000000ll);
  }
}

}  // namespace noalloc

// Error bits that calls of the allocation-free entry point recorded on the
// current device (the sticky word of its static scratch), cleared on request.
// Reads the symbol directly: allocates nothing.  0xffffffff if the read fails.
unsigned noalloc_take_device_error(bool clear) {
  unsigned v = 0;
  const size_t off = noalloc::kOffSticky;
  if (cudaMemcpyFromSymbol(&v, noalloc::g_noalloc_scratch, sizeof(v), off, cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return 0xffffffffu;
  }
  if (clear && v) {
    const unsigned zero = 0;
    if (cudaMemcpyToSymbol(noalloc::g_noalloc_scratch, &zero, sizeof(zero), off, cudaMemcpyHostToDevice) !=
        cudaSuccess)
      cudaGetLastError();
  }
  return v;
}

}  // namespace qlab

using namespace qlab;

// r = sum over the n sites of a of |a|^2 (QLA_DF3_r_veq_norm2_D semantics),
// without allocating.  Returns QLAGPU_OK or an error code (also recorded in
// qlagpu_last_error()).
extern "C" QLAB_EXPORT int qlagpu_DF3_r_veq_norm2_D_noalloc(QLA_D_Real* r, QLA_F3_DiracFermion* a, int n) {
  using namespace qlab::noalloc;
  const char* who = "qlagpu_DF3_r_veq_norm2_D_noalloc";
  if (!r || (n > 0 && !a)) {
    set_error(QLAGPU_ERR_NULLPTR, who, "NULL argument");
    return QLAGPU_ERR_NULLPTR;
  }
  if ((long long)n > kMaxSites) {
    set_error(QLAGPU_ERR_ARG, who,
              "n exceeds the static scratch of 65536 partial sums (at most 16777216 sites)");
    return QLAGPU_ERR_ARG;
  }
  const bool dev_out = is_device_ptr(r);
  cudaStream_t st = current_stream();
  if (n <= 0) {  // the reference loops zero times and stores 0
    if (dev_out) {
      if (cudaMemsetAsync(r, 0, sizeof(double), st) != cudaSuccess) {
        check_launch(who);
        return QLAGPU_ERR_LAUNCH;
      }
    } else {
      *r = 0.0;
    }
    return QLAGPU_OK;
  }
  unsigned char* base = scratch_on_current_device();
  if (!base) {
    set_error(QLAGPU_ERR_LAUNCH, who, "cudaGetSymbolAddress of the static scratch failed");
    return QLAGPU_ERR_LAUNCH;
  }
  double* result = reinterpret_cast<double*>(base + kOffResult);
  unsigned* counter = reinterpret_cast<unsigned*>(base + kOffCounter);
  unsigned* err = reinterpret_cast<unsigned*>(base + kOffErr);
  // the ticket counter and the per-call error word must start at zero; the
  // array keeps whatever the previous call (on any stream) left there
  if (cudaMemsetAsync(counter, 0, 2 * sizeof(unsigned), st) != cudaSuccess) {
    check_launch(who);
    return QLAGPU_ERR_LAUNCH;
  }

  SiteParams p = make_params(n, EQ);
  p.in[0] = op_contig(a);
  p.partials = reinterpret_cast<DD*>(base);
  p.counter = counter;
  p.err = err;
  p.result = dev_out ? static_cast<void*>(r) : static_cast<void*>(result);
  if (aligned16(a)) {
    p.stages = kStages;
    p.stage_bytes = tile_stage_bytes();
    p.tx_bytes = (unsigned)kSitesPerTile * kRecBytes;
    p.off_in[0] = 0;
    p.ntiles = (long long)n / kSitesPerTile;
    const long long grid = p.ntiles > 0 ? p.ntiles : 1;  // one tile per block; <= kMaxPartials
    const size_t smem = tile_smem_bytes();
    const void* fn = reinterpret_cast<const void*>(&site_tma_kernel<Op>);
    void* args[] = {&p};
    if (cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(kSitesPerTile + 32), args, smem, st) != cudaSuccess) {
      check_launch(who);
      return QLAGPU_ERR_LAUNCH;
    }
  } else {
    // bulk copies need 16-B alignment: one site per thread, plain loads
    long long grid = ((long long)n + 255) / 256;
    if (grid > kMaxPartials) grid = kMaxPartials;
    site_direct_kernel<Op><<<(unsigned)grid, 256, 0, st>>>(p);
  }
  if (!check_launch(who)) return QLAGPU_ERR_LAUNCH;
  noalloc_fold_error<<<1, 1, 0, st>>>(err, reinterpret_cast<unsigned*>(base + kOffSticky), dev_out ? r : nullptr);
  if (!check_launch(who)) return QLAGPU_ERR_LAUNCH;
  if (!dev_out) {
    unsigned e = 0;
    if (cudaMemcpyAsync(r, result, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(&e, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      check_launch(who);
      return QLAGPU_ERR_LAUNCH;
    }
    if (e) {
      set_error(QLAGPU_ERR_DEVICE, who, "a pipeline wait timed out");
      return QLAGPU_ERR_DEVICE;
    }
  }
  return QLAGPU_OK;
}
