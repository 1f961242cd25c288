// qla_runtime.h -- host-side runtime shared by every entry point: the current
// stream, sticky error status, per-stream reduction scratch, pointer
// classification and launch-shape tuning.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "../../include/qla_b200_runtime.h"
#include "qla_core.cuh"

// symbols of the public C API (everything else is hidden)
#define QLAB_EXPORT __attribute__((visibility("default")))

namespace qlab {

// host error codes QLAGPU_* come from the public header
void set_error(int code, const char* where, const char* detail = nullptr);
cudaStream_t current_stream();
int device_sm_count();
int current_device();

// true when p is device or managed memory (dereferenceable by kernels)
bool is_device_ptr(const void* p);

struct ReduceScratch {
  DD* partials;        // [max_blocks * 2]
  unsigned* counter;   // zero between launches
  double* result;      // [2] device result slot (used when the caller's output is host memory)
  int max_blocks;
};

// scratch for reductions issued on (current device, stream); grows to
// max_blocks.  Reductions on one stream are serialised by the stream, so one
// scratch per (device, stream) is race-free.
ReduceScratch* reduce_scratch(cudaStream_t st, int max_blocks);

// launch-shape override from the autotuner (qlagpu_tune_set): returns false
// when no override exists for this kernel id.
bool tuned_shape(const char* kernel_id, int* threads, int* stages);

// the current device's error word (device memory, zero-initialised)
unsigned* device_error_word();

// check the last launch and record an error on failure
bool check_launch(const char* where);

// Tracing: with QLA_B200_NVTX=1 in the environment (read once) every C-ABI
// entry point is an NVTX range named after its QLA function, for timeline
// tools; otherwise a range costs one predictable branch.
bool trace_enabled();
void trace_push(const char* name);
void trace_pop();
struct TraceRange {
  bool on;
  explicit TraceRange(const char* name) : on(trace_enabled()) {
    if (on) trace_push(name);
  }
  ~TraceRange() {
    if (on) trace_pop();
  }
};

}  // namespace qlab

#define QLAB_TRACE(name) ::qlab::TraceRange qlab_trace_range_(name)
