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

/* No counterpart in the reference, which dereferences every index of a
 * gather without checking (lib/perl/indirection.pl:66-101); on a GPU a bad
 * index is a device fault rather than a wrong value.  Scans the int32 index
 * stream idx[0..n) on the device for entries outside [0, nsrc) -- meant for
 * the moment an index stream is built, before any gather uses it.  Returns
 * QLAGPU_OK, or QLAGPU_ERR_ARG with *first_bad (if not NULL) set to the first
 * bad position and a message giving the count, the position and the entry.
 * Synchronises the current stream; its two result words are allocated on the
 * first call on each device. */
int qlagpu_check_index(const int *idx, long long n, long long nsrc, long long *first_bad);

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

/* Batched sequences (no counterpart in the reference): every field runs its
 * own short program of level-1 operations, all fields in one persistent
 * launch (qlagpu_batch_run; replayable from a captured CUDA graph).  A
 * program names up to 8 streams (record arrays of one field) and up to 8
 * steps.  A step reads its operands from streams or from two per-site
 * registers, leaves its result in a register and may also store it to a
 * stream.  Each step is the per-site arithmetic of the QLA_F3 function it
 * stands for, so results are bit-identical to calling those functions field
 * by field:
 *   QLAGPU_BOP_LMULT    dst (eqop) a * b  a: M (a^+ with adja), b: V, H, D or
 *                       M (b^+ with adjb, M only) -- the X_<eqop>_M{a}_times_X
 *                       family (build_qla.pl:1588-1622)
 *   QLAGPU_BOP_SPPROJ   dst (eqop) spproj(a, mu, sign); a: D, result H
 *                       (build_qla.pl:1087-1110)
 *   QLAGPU_BOP_SPRECON  dst (eqop) sprecon(a, mu, sign); a: H, result D
 *                       (build_qla.pl:1112-1135)
 *   QLAGPU_BOP_RTIMES   dst (eqop) r * a, any kind (build_qla.pl:1256-1292)
 *   QLAGPU_BOP_COPY     dst (eqop) a, any kind
 * A stream with an index reads record index[i] at site i (a gather, like the
 * `xX` forms); only IN streams gather, and no step reads a stream that the
 * launch writes (an INOUT stream reads its value from before the launch).
 * With nsrc > 0 every index is checked on the device: one outside
 * [0, nsrc) sets QLA_DEVERR_BAD_INDEX (4) in qlagpu_device_error() and the
 * site reads zeros in its place.  For peq / meq the old value comes from the
 * store stream when it is INOUT, else from the dst register.  Each stream is
 * stored by at most one step.  Bases must be 8-B aligned (16-B aligned fields
 * take the pipelined bulk-copy path), indices 4-B aligned; a malformed
 * program returns NULL with QLAGPU_ERR_ARG and a message naming the field
 * and step.  Up to 1024 fields.  The plan allocates (its device table): call
 * it outside any stream capture. */
#define QLAGPU_REC_V 0
#define QLAGPU_REC_H 1
#define QLAGPU_REC_D 2
#define QLAGPU_REC_M 3
#define QLAGPU_STREAM_IN 0
#define QLAGPU_STREAM_OUT 1
#define QLAGPU_STREAM_INOUT 2
#define QLAGPU_BOP_LMULT 0
#define QLAGPU_BOP_SPPROJ 1
#define QLAGPU_BOP_SPRECON 2
#define QLAGPU_BOP_RTIMES 3
#define QLAGPU_BOP_COPY 4
#define QLAGPU_EQ 0
#define QLAGPU_PEQ 1
#define QLAGPU_MEQ 2
#define QLAGPU_EQM 3
#define QLAGPU_REG0 8
#define QLAGPU_REG1 9
typedef struct {
  void *base;        /* device record array of this field */
  const int *index;  /* IN streams: gather index (site i reads record index[i]), or NULL */
  long long nsrc;    /* records behind a gathered stream (> 0: indices checked), else 0 */
  int kind;          /* QLAGPU_REC_V / _H / _D / _M */
  int role;          /* QLAGPU_STREAM_IN / _OUT / _INOUT */
} qlagpu_batch_stream;
typedef struct {
  int op;            /* QLAGPU_BOP_* */
  int eqop;          /* QLAGPU_EQ / _PEQ / _MEQ / _EQM */
  int a, b;          /* operands: stream 0..7 or QLAGPU_REG0 / QLAGPU_REG1 (b: LMULT only) */
  int dst;           /* QLAGPU_REG0 / QLAGPU_REG1: receives the result */
  int store;         /* stream (OUT or INOUT) that also receives the result, or -1 */
  int adja, adjb;    /* LMULT: a^+, b^+ */
  int mu, sign;      /* SPPROJ / SPRECON: mu 0..4, sign +1 / -1 */
  float r;           /* RTIMES: the real factor */
} qlagpu_batch_step;
typedef struct {
  long long n;       /* sites of this field */
  int nstreams, nsteps;
  qlagpu_batch_stream stream[8];
  qlagpu_batch_step step[8];
} qlagpu_F3_batch_program;
void *qlagpu_F3_batch_plan_program(const qlagpu_F3_batch_program *fields, int nfields);

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
