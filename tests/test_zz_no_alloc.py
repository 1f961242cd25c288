"""The allocation-free norm2 entry point, qlagpu_DF3_r_veq_norm2_D_noalloc,
called through the C-ABI.

It exists for host programs that cannot call cudaMalloc while they run (a
pool allocator that already owns the device memory, a hard memory budget):
its scratch is a static device array instead of memory allocated on first
use.  Its results must agree with the regular entry point
QLA_DF3_r_veq_norm2_D to the reductions' stated tolerance (rel <= 1e-12;
the two use different grids, hence different summation orders), on two calls
in a row (the static array keeps the previous call's contents).

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu

MAX_SITES = 65536 * 256


def _entry(qla):
    f = qla.lib().qlagpu_DF3_r_veq_norm2_D_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    return f


def _rel(a, b):
    return abs(a - b) / abs(b)


def test_noalloc_norm2_matches_regular_entry_point(qla, cuda):
    f = _entry(qla)
    g = cuda.Generator(device="cuda")
    g.manual_seed(99)
    for n in (1_000_003, 48 * 48 * 48 * 96):
        x = cuda.randn(n, 24, device="cuda", dtype=cuda.float32, generator=g)
        want = qla.DF3.r_veq_norm2_D(None, x, n)          # regular, allocating entry point
        for _ in range(2):                                 # two calls in a row
            out = ctypes.c_double(-1.0)
            rc = f(ctypes.addressof(out), x.data_ptr(), n)  # host output
            assert rc == 0, qla.last_error()
            assert _rel(out.value, want) <= 1e-12, (n, out.value, want)
            dev = cuda.full((1,), -1.0, dtype=cuda.float64, device="cuda")
            rc = f(dev.data_ptr(), x.data_ptr(), n)         # device output
            assert rc == 0, qla.last_error()
            assert _rel(float(dev.cpu()[0]), want) <= 1e-12
        del x


def test_noalloc_edge_cases(qla, cuda):
    f = _entry(qla)
    x = cuda.randn(1000, 24, device="cuda", dtype=cuda.float32)
    # small sizes and an unaligned start (direct path)
    for n, off in ((1, 0), (255, 0), (256, 0), (257, 0), (999, 1)):
        out = ctypes.c_double()
        rc = f(ctypes.addressof(out), x.data_ptr() + off * 96, n)
        assert rc == 0
        want = qla.DF3.r_veq_norm2_D(None, x.data_ptr() + off * 96, n)
        assert _rel(out.value, want) <= 1e-12, (n, off)
    out = ctypes.c_double(5.0)
    assert f(ctypes.addressof(out), x.data_ptr(), 0) == 0 and out.value == 0.0
    # beyond the static scratch: rejected before any device access
    qla.clear_error()
    assert f(ctypes.addressof(out), x.data_ptr(), MAX_SITES + 1) == 4
    code, msg = qla.last_error()
    assert code == 4 and "16777216" in msg
    qla.clear_error()
    assert qla.device_error() == 0
