// qla_runtime.cu -- host runtime of the QLA B200 library and its extra C API
// (qlagpu_*).  The reference QLA has no runtime at all: its functions are
// void, stateless and synchronous (doc/qla.tex:259-263).  A GPU drop-in needs
// a little state: the stream calls are issued on, a sticky error status
// (the QLA signatures return void), per-stream scratch for global
// reductions, and the autotuner's launch-shape table.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "../../include/qla_b200_runtime.h"
#include "qla_runtime.h"

namespace qlab {

// ---------------------------------------------------------------------------
// error status: per host thread, sticky until read/cleared
static thread_local int t_err = QLAGPU_OK;
static thread_local char t_msg[256] = {0};

void set_error(int code, const char* where, const char* detail) {
  if (t_err == QLAGPU_OK) {
    t_err = code;
    std::snprintf(t_msg, sizeof(t_msg), "%s: %s", where ? where : "qla_b200", detail ? detail : "error");
  }
}

bool check_launch(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(QLAGPU_ERR_LAUNCH, where, cudaGetErrorString(e));
    return false;
  }
  return true;
}

// ---------------------------------------------------------------------------
// stream: per host thread; default is the legacy default stream, which makes
// every call ordered with the caller's other default-stream work (a
// synchronous-looking drop-in).
static thread_local cudaStream_t t_stream = nullptr;

cudaStream_t current_stream() { return t_stream; }

int current_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

int device_sm_count() {
  static std::mutex mu;
  static std::map<int, int> cache;
  const int d = current_device();
  std::lock_guard<std::mutex> g(mu);
  auto it = cache.find(d);
  if (it != cache.end()) return it->second;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d) != cudaSuccess || sms <= 0) sms = 1;
  cache[d] = sms;
  return sms;
}

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // unregistered host memory on older runtimes
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// ---------------------------------------------------------------------------
// per-(device, stream) reduction scratch and per-device error word
namespace {
struct DevState {
  unsigned* err = nullptr;
};
std::mutex g_mu;
std::map<int, DevState> g_dev;
std::map<std::pair<int, cudaStream_t>, ReduceScratch> g_scratch;
}  // namespace

unsigned* device_error_word() {
  const int d = current_device();
  std::lock_guard<std::mutex> g(g_mu);
  DevState& s = g_dev[d];
  if (!s.err) {
    unsigned* p = nullptr;
    if (cudaMalloc(&p, sizeof(unsigned)) != cudaSuccess) {
      cudaGetLastError();
      set_error(QLAGPU_ERR_ALLOC, "device_error_word", "cudaMalloc failed");
      return nullptr;
    }
    cudaMemset(p, 0, sizeof(unsigned));
    s.err = p;
  }
  return s.err;
}

ReduceScratch* reduce_scratch(cudaStream_t st, int max_blocks) {
  const int d = current_device();
  std::lock_guard<std::mutex> g(g_mu);
  ReduceScratch& rs = g_scratch[std::make_pair(d, st)];
  if (rs.max_blocks >= max_blocks) return &rs;
  // (re)allocate: [partials (2 DD per block)] [result: 2 doubles] [counter]
  if (rs.partials) {
    cudaStreamSynchronize(st);
    cudaFree(rs.partials);
  }
  size_t bytes = sizeof(DD) * 2 * (size_t)max_blocks + 2 * sizeof(double) + 256;
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    rs = ReduceScratch{};
    set_error(QLAGPU_ERR_ALLOC, "reduce_scratch", "cudaMalloc failed");
    return nullptr;
  }
  cudaMemset(p, 0, bytes);
  rs.partials = static_cast<DD*>(p);
  rs.result = reinterpret_cast<double*>(static_cast<char*>(p) + sizeof(DD) * 2 * (size_t)max_blocks);
  rs.counter = reinterpret_cast<unsigned*>(reinterpret_cast<char*>(rs.result) + 2 * sizeof(double));
  rs.max_blocks = max_blocks;
  return &rs;
}

// ---------------------------------------------------------------------------
// autotuner table: kernel id -> (threads, stages)
namespace {
std::mutex g_tune_mu;
std::map<std::string, std::pair<int, int>> g_tune;
std::atomic<int> g_tune_count{0};
}  // namespace

// The shipped table (tune_b200.txt beside the package, written by
// `python -m qla_b200.tune` on a B200) or the file named by $QLA_B200_TUNE is
// read once, at the first launch.  Lines: "<kernel id> <threads> <stages>".
static std::once_flag g_tune_once;

static void load_tune_file() {
  std::string path;
  if (const char* env = std::getenv("QLA_B200_TUNE")) {
    path = env;
  } else {
    Dl_info info;
    if (dladdr(reinterpret_cast<void*>(&load_tune_file), &info) && info.dli_fname) {
      std::string so = info.dli_fname;
      size_t k = so.rfind('/');
      std::string dir = (k == std::string::npos) ? std::string(".") : so.substr(0, k);
      path = dir + "/../tune_b200.txt";
    }
  }
  if (path.empty() || path == "none") return;
  std::ifstream f(path);
  if (!f) return;
  std::string line;
  std::lock_guard<std::mutex> g(g_tune_mu);
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream ss(line);
    std::string id;
    int t = 0, st = 0;
    if (ss >> id >> t >> st && (t == 64 || t == 128 || t == 256) && st >= 2 && st <= 8)
      g_tune[id] = std::make_pair(t, st);
  }
  g_tune_count.store((int)g_tune.size());
}

bool tuned_shape(const char* kernel_id, int* threads, int* stages) {
  std::call_once(g_tune_once, load_tune_file);
  if (g_tune_count.load(std::memory_order_relaxed) == 0 || !kernel_id) return false;
  std::lock_guard<std::mutex> g(g_tune_mu);
  auto it = g_tune.find(kernel_id);
  if (it == g_tune.end()) {
    // fall back from "<id>:<operand modes>" to the family-wide "<id>"
    const char* colon = std::strchr(kernel_id, ':');
    if (!colon) return false;
    it = g_tune.find(std::string(kernel_id, colon - kernel_id));
    if (it == g_tune.end()) return false;
  }
  *threads = it->second.first;
  *stages = it->second.second;
  return true;
}

// ---------------------------------------------------------------------------
// Self-test of the failure path: one block waits on an mbarrier phase that
// nothing will ever complete (one expected arrival, none made), with a short
// time limit.  The wait must give up, raise QLA_DEVERR_MBAR_TIMEOUT in the
// error word and return, leaving the context usable.
__global__ void wait_timeout_selftest_kernel(unsigned* err, unsigned long long limit_ns, int* gave_up) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (threadIdx.x == 0) *gave_up = mbar_wait_bounded(&bar, 0u, err, limit_ns) ? 0 : 1;
}

bool trace_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("QLA_B200_NVTX");
    return e && e[0] && e[0] != '0';
  }();
  return on;
}
void trace_push(const char* name) { nvtxRangePushA(name); }
void trace_pop() { nvtxRangePop(); }

// error bits recorded by the allocation-free entry point on the current
// device (defined in qla_noalloc.cu); allocates nothing
unsigned noalloc_take_device_error(bool clear);

}  // namespace qlab

// ===========================================================================
// extra C API
using namespace qlab;

extern "C" {

QLAB_EXPORT int qlagpu_last_error(void) { return t_err; }

QLAB_EXPORT const char* qlagpu_last_error_string(void) { return t_err == QLAGPU_OK ? "" : t_msg; }

QLAB_EXPORT void qlagpu_clear_error(void) {
  t_err = QLAGPU_OK;
  t_msg[0] = 0;
}

QLAB_EXPORT void qlagpu_set_stream(void* stream) { t_stream = static_cast<cudaStream_t>(stream); }

QLAB_EXPORT void* qlagpu_get_stream(void) { return static_cast<void*>(t_stream); }

// The regular entry points' error word (allocated by the first launch on a
// device; no kernel can have written to a word that does not exist yet, so it
// is not allocated here) OR the sticky word of the allocation-free entry
// point's static scratch.  Allocates nothing.
QLAB_EXPORT unsigned qlagpu_device_error(int clear) {
  unsigned* w = nullptr;
  {
    const int d = current_device();
    std::lock_guard<std::mutex> g(g_mu);
    w = g_dev[d].err;
  }
  unsigned v = 0;
  if (cudaStreamSynchronize(t_stream) != cudaSuccess ||
      (w && cudaMemcpy(&v, w, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess)) {
    check_launch("qlagpu_device_error");
    return 0xffffffffu;
  }
  if (clear && v) cudaMemset(w, 0, sizeof(unsigned));
  const unsigned nv = noalloc_take_device_error(clear != 0);
  if (nv == 0xffffffffu) {
    set_error(QLAGPU_ERR_LAUNCH, "qlagpu_device_error", "reading the allocation-free scratch failed");
    return 0xffffffffu;
  }
  v |= nv;
  if (v) set_error(QLAGPU_ERR_DEVICE, "qlagpu_device_error", "a kernel reported an error");
  return v;
}

QLAB_EXPORT int qlagpu_synchronize(void) {
  if (cudaStreamSynchronize(t_stream) != cudaSuccess) {
    check_launch("qlagpu_synchronize");
    return t_err;
  }
  return QLAGPU_OK;
}

QLAB_EXPORT int qlagpu_tune_set(const char* kernel_id, int threads, int stages) {
  std::call_once(g_tune_once, load_tune_file);
  if (!kernel_id || !(threads == 64 || threads == 128 || threads == 256) || stages < 2 || stages > 8) {
    set_error(QLAGPU_ERR_ARG, "qlagpu_tune_set", "threads must be 64/128/256 and stages 2..8");
    return QLAGPU_ERR_ARG;
  }
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune[kernel_id] = std::make_pair(threads, stages);
  g_tune_count.store((int)g_tune.size());
  return QLAGPU_OK;
}

QLAB_EXPORT void qlagpu_tune_clear(void) {
  std::call_once(g_tune_once, load_tune_file);  // a later first launch must not reload it
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune.clear();
  g_tune_count.store(0);
}

QLAB_EXPORT int qlagpu_sm_count(void) { return device_sm_count(); }

// Runs the failure-path self-test with a wait limit of limit_us microseconds
// (1..1000000).  Returns 1 when the wait gave up and the error word carries
// the timeout bit (which is then cleared), 0 when it did not, or a negative
// value when the test could not run.
QLAB_EXPORT int qlagpu_selftest_wait_timeout(int limit_us) {
  if (limit_us < 1 || limit_us > 1000000) {
    set_error(QLAGPU_ERR_ARG, "qlagpu_selftest_wait_timeout", "limit_us must be in 1..1000000");
    return -1;
  }
  unsigned* err = device_error_word();
  if (!err) return -2;
  int* flag = nullptr;
  if (cudaMalloc(&flag, sizeof(int)) != cudaSuccess) {
    check_launch("qlagpu_selftest_wait_timeout");
    return -2;
  }
  cudaMemset(flag, 0, sizeof(int));
  cudaMemset(err, 0, sizeof(unsigned));
  wait_timeout_selftest_kernel<<<1, 32, 0, t_stream>>>(err, 1000ull * (unsigned long long)limit_us, flag);
  int gave_up = 0;
  unsigned bits = 0;
  const bool ok = check_launch("qlagpu_selftest_wait_timeout") &&
                  cudaMemcpy(&gave_up, flag, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess &&
                  cudaMemcpy(&bits, err, sizeof(unsigned), cudaMemcpyDeviceToHost) == cudaSuccess;
  cudaFree(flag);
  if (!ok) return -3;
  cudaMemset(err, 0, sizeof(unsigned));
  return (gave_up == 1 && (bits & QLA_DEVERR_MBAR_TIMEOUT)) ? 1 : 0;
}

QLAB_EXPORT const char* qlagpu_version(void) { return "qla_b200 0.1 (QLA 1.9.0 level-1 API, sm_100a)"; }

}  // extern "C"
