/*
 * qla_b200_runtime.h -- the small runtime API that a GPU drop-in of QLA needs
 * and the reference does not have.
 *
 * Reference behaviour being extended: every QLA function is void, synchronous,
 * stateless and works on host memory (doc/qla.tex:259-263).  Here:
 *  - array arguments are device (or managed) pointers; pointer arrays (`pX`
 *    arguments) are device arrays of device pointers;
 *  - scalar inputs (`QLA_F_Real *a` ...) may be host or device pointers: a host
 *    scalar is read at call time, a device scalar is read by the kernel;
 *  - reduction outputs may be host or device pointers: a host output makes the
 *    call synchronous (the reference's semantics), a device output keeps it
 *    asynchronous on the current stream;
 *  - calls are issued on a per-host-thread current stream (default: the legacy
 *    default stream);
 *  - errors are recorded in a sticky per-thread status, because the QLA
 *    signatures return void.
 */
#ifndef QLA_B200_RUNTIME_H
#define QLA_B200_RUNTIME_H
#include "qla_b200_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* error codes of qlagpu_last_error() */
#define QLAGPU_OK 0
#define QLAGPU_ERR_NULLPTR 1
#define QLAGPU_ERR_LAUNCH 2
#define QLAGPU_ERR_ALLOC 3
#define QLAGPU_ERR_ARG 4
#define QLAGPU_ERR_DEVICE 5
#define QLAGPU_ERR_NOT_DEVICE 6

/* sticky status of this host thread (first error since the last clear) */
int qlagpu_last_error(void);
const char *qlagpu_last_error_string(void);
void qlagpu_clear_error(void);

/* stream subsequent calls of this host thread are issued on (cudaStream_t) */
void qlagpu_set_stream(void *stream);
void *qlagpu_get_stream(void);
/* synchronise the current stream; returns the sticky status */
int qlagpu_synchronize(void);

/* synchronise, then return the device error word (bit 1: a pipeline wait gave
 * up; 2: draining copies gave up; 8: an iterative matrix function hit its
 * iteration cap), together with the bits recorded by
 * qlagpu_DF3_r_veq_norm2_D_noalloc; clear != 0 resets both.  Allocates no
 * device memory. */
unsigned qlagpu_device_error(int clear);

/* autotuner: launch shape (threads per block = sites per tile: 64/128/256,
 * pipeline stages: 2..8) for one kernel id, as reported by
 * qla_b200.tune; qlagpu_tune_clear() restores the built-in heuristic */
int qlagpu_tune_set(const char *kernel_id, int threads, int stages);
void qlagpu_tune_clear(void);

int qlagpu_sm_count(void);

/* failure-path self-test: a kernel waits on a barrier that nothing completes,
 * with a limit of limit_us microseconds; returns 1 when the wait gave up and
 * reported the timeout (the context stays usable), 0 otherwise, < 0 when the
 * test could not run */
int qlagpu_selftest_wait_timeout(int limit_us);
const char *qlagpu_version(void);

/* periodic neighbour table on the device: idx[i] = the lexicographic site
 * (x0 fastest) of x(i) + sign * e_mu on the nd-dimensional torus dims[];
 * n = prod(dims).  This is the int32 index stream the `xX` gathers take. */
void qlagpu_shift_index(int *idx, int nd, const int *dims, int mu, int sign);

/* Batched uneven-volume execution (no counterpart in the reference, which
 * handles one field per call).  Per field f and site i < n:
 *     r[i] = u[i] * u2[nbr[i]]   -- QLA_F3_M_eq_M_times_xM
 *     w[i] = r[i] * v[i]         -- QLA_F3_V_veq_M_times_V
 * for all fields in one persistent launch; results are bit-identical to the
 * two calls per field.  qlagpu_F3_batch_plan copies the field table to the
 * device (it allocates; call it outside any stream capture);
 * qlagpu_batch_run is a single kernel launch on the current stream with no
 * allocation or host synchronisation; qlagpu_batch_destroy frees the plan.
 * Up to 1024 fields; fields whose arrays are not 16-B aligned take the
 * plain-load path. */
typedef struct {
  QLA_F3_ColorMatrix *r;
  QLA_F3_ColorMatrix *u;
  QLA_F3_ColorMatrix *u2;
  int *nbr;
  QLA_F3_ColorVector *w;
  QLA_F3_ColorVector *v;
  long long n;
} qlagpu_F3_batch_field;
void *qlagpu_F3_batch_plan(const qlagpu_F3_batch_field *fields, int nfields);
int qlagpu_batch_run(void *plan);
void qlagpu_batch_destroy(void *plan);

/* No counterpart in the reference (QLA never touches device memory).
 * QLA_DF3_r_veq_norm2_D for callers that cannot allocate device memory while
 * they run -- e.g. a program whose own pool allocator reserved the GPU's
 * memory up front, or one under a hard memory budget: the regular reductions
 * allocate their scratch on first use, this one allocates nothing.  Its
 * scratch is a static 1 MiB device array held by every GPU that loads the
 * library until the process exits; it limits n to 16,777,216 sites (larger n
 * return QLAGPU_ERR_ARG).  The first call on a device looks the array up
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * All calls share the array: calls that overlap on the GPU (e.g. on two
 * streams at once) race and give wrong results.  r may be a host pointer
 * (the call synchronises and returns QLAGPU_ERR_DEVICE if a pipeline wait
 * gave up) or a device pointer (the call stays asynchronous; if a wait gave
 * up, *r is set to NaN and qlagpu_device_error() reports the bits).  Returns
 * QLAGPU_OK or an error code. */
int qlagpu_DF3_r_veq_norm2_D_noalloc(QLA_D_Real *r, QLA_F3_DiracFermion *a, int n);

#ifdef __cplusplus
}
#endif

#endif /* QLA_B200_RUNTIME_H */
