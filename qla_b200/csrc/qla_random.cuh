// qla_random.cuh -- QLA's per-site random-number generator on the device:
// uniform fills (R_*_random_S), gaussian fills of every field type
// (X_*_gaussian_S), seeding from an integer field (S_*_seed_i_I) and copies /
// masked copies of the state fields (S_*_S, S_*_S_mask_I).
//
// The generator is the reference's (lib/random/QLA_random.c:18-36): an
// exclusive-or of a 24-bit feedback shift register over seven words and a
// 32-bit congruential generator with a per-site multiplier, scaled by 2^-24.
// All of it is integer arithmetic and one exact float product, so uniform
// deviates and the states left behind are bit-identical to the reference.
// Gaussian deviates follow lib/random/QLA_gaussian.c:19-55: Box-Muller in
// double (default) or MILC's polar method (QLA_use_milc_gaussian != 0, the
// spare deviate kept in the state's addend / scale words), rounded to float.
// Their double log / cos / sqrt are CUDA's: sqrt is correctly rounded; log
// and cos may differ from the host libm in the last place of the double,
// which changes the float result only when it falls within that distance of
// a float rounding boundary.
//
// Fills run one thread per site (the state is sequential within a site) and
// generate the record's values in the reference's order: for each complex
// element the real part, then the imaginary part.  Seeding follows
// lib/random/QLA_seed_random.c:13-36.
#pragma once
#include "qla_ewise.cuh"

extern "C" int QLA_use_milc_gaussian;

namespace qlab {

inline int rng_milc_flag() { return QLA_use_milc_gaussian != 0 ? 1 : 0; }

struct RandState {
  unsigned r0, r1, r2, r3, r4, r5, r6, multiplier, addend, ic_state;
  float scale;
};
static_assert(sizeof(RandState) == 44, "QLA_RandomState layout");

// QLA_random: uniform on [0, 1)
__host__ __device__ __forceinline__ float rng_uniform(RandState& s) {
  const int t = (int)((((s.r5 >> 7) | (s.r6 << 17)) ^ ((s.r4 >> 1) | (s.r5 << 23))) & 0xffffffu);
  s.r6 = s.r5;
  s.r5 = s.r4;
  s.r4 = s.r3;
  s.r3 = s.r2;
  s.r2 = s.r1;
  s.r1 = s.r0;
  s.r0 = (unsigned)t;
  const unsigned c = s.ic_state * s.multiplier + 12345u;
  s.ic_state = c;
  // (c >> 8) & 0xffffff keeps bits 8..31 whatever the shift fills in
  return (1.0f / (float)0x1000000) * (float)(t ^ (int)((c >> 8) & 0xffffffu));
}

// QLA_seed_random(s, seed, index)
__host__ __device__ __forceinline__ void rng_seed(RandState& s, int seed, int index) {
  const unsigned m = 69607u + 8u * (unsigned)index;
  unsigned x = (unsigned)seed;
  unsigned w[8];
  for (int j = 0; j < 8; j++) {
    x = m * x + 12345u;
    w[j] = x;
  }
  s.r0 = (w[0] >> 8) & 0xffffffu;
  s.r1 = (w[1] >> 8) & 0xffffffu;
  s.r2 = (w[2] >> 8) & 0xffffffu;
  s.r3 = (w[3] >> 8) & 0xffffffu;
  s.r4 = (w[4] >> 8) & 0xffffffu;
  s.r5 = (w[5] >> 8) & 0xffffffu;
  s.r6 = (w[6] >> 8) & 0xffffffu;
  s.ic_state = w[7];
  s.multiplier = 100005u + 8u * (unsigned)index;
  s.addend = 12345u;
  s.scale = (float)(1.0 / (double)(float)0x1000000);
}

// the polar method's rejection loop ends with probability pi/4 per pass; the
// device form gives up (and reports it) after this many passes
constexpr int kPolarMaxPasses = 4096;

// QLA_gaussian; *bad is set when the polar method ran out of passes
__device__ __forceinline__ float rng_gaussian(RandState& s, int milc, unsigned* bad) {
  if (milc) {
    if (s.addend != 0u) {
      s.addend = 0u;
      double v1 = 0.0, v2 = 0.0, rsq = 0.0;
      int pass = 0;
      do {
        v1 = (double)rng_uniform(s);
        v2 = (double)rng_uniform(s);
        v1 = __dsub_rn(__dmul_rn(2.0, v1), 1.0);
        v2 = __dsub_rn(__dmul_rn(2.0, v2), 1.0);
        rsq = __dadd_rn(__dmul_rn(v1, v1), __dmul_rn(v2, v2));
      } while ((rsq >= 1.0 || rsq == 0.0) && ++pass < kPolarMaxPasses);
      if (pass >= kPolarMaxPasses) *bad = 1u;
      const double fac = __dsqrt_rn(__ddiv_rn(__dmul_rn(-2.0, log(rsq)), rsq));
      s.scale = (float)__dmul_rn(v1, fac);
      return (float)__dmul_rn(v2, fac);
    }
    s.addend = 1u;
    return s.scale;
  }
  const double v = (double)rng_uniform(s);
  const double p = __dmul_rn(__dmul_rn((double)rng_uniform(s), 2.0), 3.14159265358979323846);
  const double r = __dsqrt_rn(__dmul_rn(2.0, -log(__dadd_rn(v, 1e-307))));
  return (float)__dmul_rn(r, cos(p));
}

__device__ __forceinline__ RandState rng_load(const void* p) {
  const unsigned* w = static_cast<const unsigned*>(p);
  RandState s;
  s.r0 = w[0];
  s.r1 = w[1];
  s.r2 = w[2];
  s.r3 = w[3];
  s.r4 = w[4];
  s.r5 = w[5];
  s.r6 = w[6];
  s.multiplier = w[7];
  s.addend = w[8];
  s.ic_state = w[9];
  s.scale = __uint_as_float(w[10]);
  return s;
}

__device__ __forceinline__ void rng_store(void* p, const RandState& s) {
  unsigned* w = static_cast<unsigned*>(p);
  w[0] = s.r0;
  w[1] = s.r1;
  w[2] = s.r2;
  w[3] = s.r3;
  w[4] = s.r4;
  w[5] = s.r5;
  w[6] = s.r6;
  w[7] = s.multiplier;
  w[8] = s.addend;
  w[9] = s.ic_state;
  w[10] = __float_as_uint(s.scale);
}

__device__ __forceinline__ void* state_ptr(const Opnd& o, long long k) {
  return (o.mode == OM_PTR) ? const_cast<void*>(o.ptrs[k])
                            : static_cast<void*>(static_cast<char*>(const_cast<void*>(o.base)) + k * 44);
}

struct RngParams {
  void* out;
  Opnd s;          // state field (read and written)
  Opnd m;          // QLA_Int field (mask / seeding index)
  const int* gang;
  long long n;
  int nreal;       // reals per output record (1 for a real field)
  int gauss;       // 0: uniform, 1: gaussian
  int milc;
  int seed;
  unsigned* err;
};

// uniform / gaussian fill of a field of R records (nreal reals each)
template <typename R>
__global__ void __launch_bounds__(128) rng_fill_kernel(const RngParams p) {
  unsigned bad = 0u;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < p.n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long k = p.gang ? (long long)p.gang[i] : i;
    void* sp = state_ptr(p.s, k);
    RandState s = rng_load(sp);
    R* out = static_cast<R*>(p.out) + k * p.nreal;
    for (int c = 0; c < p.nreal; c++) out[c] = (R)(p.gauss ? rng_gaussian(s, p.milc, &bad) : rng_uniform(s));
    rng_store(sp, s);
  }
  if (bad) raise_dev_error(p.err, QLA_DEVERR_RNG);
}

// S_*_seed_i_I: state k = QLA_seed_random(seed, a[k])
static __global__ void __launch_bounds__(256) rng_seed_kernel(const RngParams p) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < p.n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long k = p.gang ? (long long)p.gang[i] : i;
    const int idx = (p.m.mode == OM_PTR) ? *static_cast<const int*>(p.m.ptrs[k]) : static_cast<const int*>(p.m.base)[k];
    RandState s;
    rng_seed(s, p.seed, idx);
    rng_store(static_cast<char*>(p.out) + k * 44, s);
  }
}

// S_*_S and S_*_S_mask_I: 11 words per state, one thread per word
static __global__ void __launch_bounds__(256) rng_copy_kernel(const RngParams p, int masked) {
  const long long total = p.n * 11;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const long long i = g / 11;
    const int w = (int)(g - i * 11);
    const long long k = p.gang ? (long long)p.gang[i] : i;
    if (masked) {
      const int mv =
          (p.m.mode == OM_PTR) ? *static_cast<const int*>(p.m.ptrs[k]) : static_cast<const int*>(p.m.base)[k];
      if (!mv) continue;
    }
    static_cast<unsigned*>(p.out)[k * 11 + w] = static_cast<const unsigned*>(state_ptr(p.s, k))[w];
  }
}

inline bool rng_prep(const char* kid, RngParams& p, void* r, Opnd s, const int* gang, int n) {
  if (n <= 0) return false;
  if (!r || !opnd_ok(s)) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return false;
  }
  std::memset(&p, 0, sizeof(p));
  p.out = r;
  p.s = s;
  p.gang = gang;
  p.n = n;
  p.err = device_error_word();
  return true;
}

inline unsigned rng_grid(long long total, int threads) {
  const long long cap = (long long)device_sm_count() * 16;
  long long grid = (total + threads - 1) / threads;
  if (grid > cap) grid = cap;
  return (unsigned)(grid < 1 ? 1 : grid);
}

// r (nreal reals per record of R) = uniform (gauss 0) or gaussian deviates
template <typename R>
inline void rng_fill(const char* kid, int nreal, int gauss, void* r, Opnd s, const int* gang, int n) {
  RngParams p;
  if (!rng_prep(kid, p, r, s, gang, n)) return;
  p.nreal = nreal;
  p.gauss = gauss;
  p.milc = rng_milc_flag();
  rng_fill_kernel<R><<<rng_grid(n, 128), 128, 0, current_stream()>>>(p);
  check_launch(kid);
}

// fills of a real field (REAL) or of records of NE complex numbers
template <typename R, int NE, bool REAL>
inline void api_rng_fill(const char* kid, int gauss, void* r, Opnd s, const int* gang, int n) {
  rng_fill<R>(kid, REAL ? 1 : 2 * NE, gauss, r, s, gang, n);
}

// the same with nc colours (records of ne complex numbers)
template <typename R>
inline void api_rng_fill_n(const char* kid, int nc, int ne, int gauss, void* r, Opnd s, const int* gang, int n) {
  if (nc < 1 || nc > 64) {
    set_error(QLAGPU_ERR_ARG, kid, "nc outside 1..64");
    return;
  }
  rng_fill<R>(kid, 2 * ne, gauss, r, s, gang, n);
}

inline void api_rng_seed(const char* kid, void* r, int seed, Opnd a, const int* gang, int n) {
  RngParams p;
  if (!rng_prep(kid, p, r, Opnd{}, gang, n)) return;
  if (!opnd_ok(a)) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  p.m = a;
  p.seed = seed;
  rng_seed_kernel<<<rng_grid(n, 256), 256, 0, current_stream()>>>(p);
  check_launch(kid);
}

inline void api_rng_copy(const char* kid, void* r, Opnd a, Opnd mask, bool masked, const int* gang, int n) {
  RngParams p;
  if (!rng_prep(kid, p, r, a, gang, n)) return;
  if (masked && !opnd_ok(mask)) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  p.m = mask;
  rng_copy_kernel<<<rng_grid((long long)n * 11, 256), 256, 0, current_stream()>>>(p, masked ? 1 : 0);
  check_launch(kid);
}

}  // namespace qlab
