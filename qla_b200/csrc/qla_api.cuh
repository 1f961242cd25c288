// qla_api.cuh -- host templates behind the generated extern "C" QLA entry
// points: argument checks, operand descriptors, host/device scalar and
// reduction-output handling, then the engine launch.
#pragma once
#include "qla_launch.cuh"
#include "qla_ops.cuh"

namespace qlab {

inline bool opnd_ok(const Opnd& o) {
  switch (o.mode) {
    case OM_CONTIG: return o.base != nullptr;
    case OM_PTR: return o.ptrs != nullptr;
    case OM_IDX: return o.base != nullptr && o.idx != nullptr;
    default: return true;
  }
}

template <class OP>
inline void api_map(const char* kid, void* r, Opnd a, Opnd b, const int* gang, int n, int eqop, int mu = 0,
                    int sign = 1) {
  if (n <= 0) return;
  if (!r || !opnd_ok(a) || (OP::NIN > 1 && !opnd_ok(b))) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL array argument");
    return;
  }
  SiteParams p = make_params(n, eqop);
  p.in[0] = a;
  if (OP::NIN > 1) p.in[1] = b;
  p.out = r;
  p.gang = gang;
  p.mu = mu;
  p.sign = sign;
  SiteLauncher<OP>::run(p, kid);
}

// scalar-coefficient maps (r (eqop) a * b with `a` passed by pointer)
template <class OP, typename S>
inline void api_scalar_map(const char* kid, void* r, const S* a, Opnd b, const int* gang, int n, int eqop) {
  if (n <= 0) return;
  if (!r || !a || !opnd_ok(b)) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  SiteParams p = make_params(n, eqop);
  p.in[0] = b;
  p.out = r;
  p.gang = gang;
  if (is_device_ptr(a))
    p.sptr = a;
  else
    p.sval = static_cast<double>(*a);
  SiteLauncher<OP>::run(p, kid);
}

// global reductions: r may be host (synchronous) or device (asynchronous)
template <class OP>
inline void api_reduce(const char* kid, void* r, size_t rbytes, Opnd a, Opnd b, const int* gang, int n) {
  if (!r || (n > 0 && (!opnd_ok(a) || (OP::NIN > 1 && !opnd_ok(b))))) {
    set_error(QLAGPU_ERR_NULLPTR, kid, "NULL argument");
    return;
  }
  SiteParams p = make_params(n, EQ);
  p.in[0] = a;
  if (OP::NIN > 1) p.in[1] = b;
  p.gang = gang;
  if (is_device_ptr(r)) {
    p.result = r;
    SiteLauncher<OP>::run(p, kid, nullptr, rbytes);
  } else {
    SiteLauncher<OP>::run(p, kid, r, rbytes);
  }
}

}  // namespace qlab
