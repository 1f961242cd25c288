// qla_random_host.cu -- the reference's host functions on ONE random-number
// state in host memory (lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55,
// QLA_seed_random.c:13-36) and the QLA_use_milc_gaussian switch
// (QLA_gaussian.c:9), so that programs that seed or draw on the host link
// against this library unchanged.  They share rng_uniform / rng_seed with the
// device fills; the gaussian uses the host libm, as the reference does.  The
// field fills (X_*_gaussian_S, R_*_random_S) run on the device.
#include <cmath>

#include "../../include/qla_b200_types.h"
#include "qla_runtime.h"
#include "qla_random.cuh"

extern "C" {

QLAB_EXPORT int QLA_use_milc_gaussian = 0;

QLAB_EXPORT QLA_F_Real QLA_random(QLA_RandomState* prn_pt) {
  return qlab::rng_uniform(*reinterpret_cast<qlab::RandState*>(prn_pt));
}

QLAB_EXPORT void QLA_seed_random(QLA_RandomState* prn_pt, int seed, QLA_Int index) {
  qlab::rng_seed(*reinterpret_cast<qlab::RandState*>(prn_pt), seed, index);
}

QLAB_EXPORT QLA_F_Real QLA_gaussian(QLA_RandomState* rs) {
  qlab::RandState& s = *reinterpret_cast<qlab::RandState*>(rs);
  if (QLA_use_milc_gaussian) {
    if (s.addend != 0u) {
      s.addend = 0u;
      double v1, v2, rsq;
      do {
        v1 = (double)qlab::rng_uniform(s);
        v2 = (double)qlab::rng_uniform(s);
        v1 = 2.0 * v1 - 1.0;
        v2 = 2.0 * v2 - 1.0;
        rsq = v1 * v1 + v2 * v2;
      } while ((rsq >= 1.0) || (rsq == 0.0));
      const double fac = std::sqrt(-2.0 * std::log(rsq) / rsq);
      s.scale = (float)(v1 * fac);
      return (float)(v2 * fac);
    }
    s.addend = 1u;
    return s.scale;
  }
  const double v = qlab::rng_uniform(s);
  const double p = qlab::rng_uniform(s) * 2. * 3.14159265358979323846;
  const double r = std::sqrt(2. * (-std::log(v + 1e-307)));
  return (QLA_F_Real)(r * std::cos(p));
}

}  // extern "C"
