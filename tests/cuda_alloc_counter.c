/* Test helper, preloaded (LD_PRELOAD) into a child process by
 * tests/test_zz_no_alloc.py: it stands between the process and the CUDA
 * runtime library, counts every call of the runtime's allocation and release
 * functions, and logs the block size of every kernel launch, then forwards
 * each call unchanged to the real runtime (dlsym RTLD_NEXT).  It lets a test
 * show that an entry point allocates and frees nothing, its first call on a
 * device included, and which kernel path a call took. */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <stddef.h>

typedef int cudaError_t;
typedef struct {
  unsigned x, y, z;
} dim3_t; /* the runtime's dim3: three unsigned, passed by value */

static volatile long g_allocs;
static volatile int g_nlaunch;
static unsigned g_launch_block[256];

long qla_test_alloc_calls(void) { return g_allocs; }
int qla_test_launches(unsigned *block_x, int max) {
  int n = g_nlaunch < max ? g_nlaunch : max;
  for (int i = 0; i < n; i++) block_x[i] = g_launch_block[i];
  return g_nlaunch;
}
void qla_test_reset_launches(void) { g_nlaunch = 0; }

static void *next_fn(const char *name) { return dlsym(RTLD_NEXT, name); }

#define COUNTED(name, params, args)                           \
  cudaError_t name params {                                   \
    static cudaError_t(*real) params;                         \
    if (!real) real = (cudaError_t(*) params)next_fn(#name);  \
    __sync_fetch_and_add(&g_allocs, 1);                       \
    return real args;                                         \
  }

COUNTED(cudaMalloc, (void **p, size_t n), (p, n))
COUNTED(cudaMallocAsync, (void **p, size_t n, void *s), (p, n, s))
COUNTED(cudaMallocFromPoolAsync, (void **p, size_t n, void *pool, void *s), (p, n, pool, s))
COUNTED(cudaMallocManaged, (void **p, size_t n, unsigned f), (p, n, f))
COUNTED(cudaMallocHost, (void **p, size_t n), (p, n))
COUNTED(cudaHostAlloc, (void **p, size_t n, unsigned f), (p, n, f))
COUNTED(cudaMallocPitch, (void **p, size_t *pitch, size_t w, size_t h), (p, pitch, w, h))
COUNTED(cudaFree, (void *p), (p))
COUNTED(cudaFreeAsync, (void *p, void *s), (p, s))
COUNTED(cudaFreeHost, (void *p), (p))

cudaError_t cudaLaunchKernel(const void *fn, dim3_t grid, dim3_t block, void **args, size_t smem, void *stream) {
  static cudaError_t (*real)(const void *, dim3_t, dim3_t, void **, size_t, void *);
  if (!real) real = (cudaError_t(*)(const void *, dim3_t, dim3_t, void **, size_t, void *))next_fn("cudaLaunchKernel");
  int k = __sync_fetch_and_add(&g_nlaunch, 1);
  if (k < 256) g_launch_block[k] = block.x;
  return real(fn, grid, block, args, smem, stream);
}
