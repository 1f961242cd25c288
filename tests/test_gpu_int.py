"""GPU parity of all QLA_I_ integer entry points (v and x variants, every
eqop, pointer operands) against the oracle, bit-exact, through the C-ABI;
plus the 16-B vectorised path on a large field and an unaligned start."""
import ctypes

import numpy as np
import pytest

import qla_testlib as T

pytestmark = pytest.mark.gpu


def test_all_int_entry_points(qla, cuda):
    rng = np.random.default_rng(31)
    n, ns = 3001, 3200
    ins = T.int_inputs(rng, n, ns)
    names = [e["name"] for e in qla.manifest() if e["name"].startswith("QLA_I_")]
    assert len(names) == 238
    dev = {id(v): T.to_dev(v) for v in ins.values()}
    keep = []

    def arr(a):
        t = dev.get(id(a))
        if t is None:
            t = T.to_dev(a)
            keep.append(t)
        return t

    def ptrs(a, idx):
        t = T.to_dev(dev[id(a)].data_ptr() + idx.astype(np.int64) * 4)
        keep.append(t)
        return t

    L = qla.lib()
    bad = []
    for name in names:
        r = T.to_dev(ins["r0"])
        args = T.int_call_args(name, ins, n, r, arr, ptrs)
        cargs = [a.data_ptr() if hasattr(a, "data_ptr") else a for a in args]
        fn = getattr(L, name)
        fn.restype = None
        fn(*[ctypes.c_int(a) if isinstance(a, int) and a == n and i == len(cargs) - 1 else ctypes.c_void_p(a)
             for i, a in enumerate(cargs)])
        qla.check(name)
        if not np.array_equal(T.to_host(r), T.ora_int(name, ins, n)):
            bad.append(name)
    assert not bad, bad[:10]


def test_int_vector_path_large_and_unaligned(qla, cuda):
    rng = np.random.default_rng(32)
    n = 5_000_011
    a = rng.integers(-2**31, 2**31 - 1, n + 1, dtype=np.int64).astype(np.int32)
    b = rng.integers(1, 32, n + 1).astype(np.int32)
    for off in (0, 1):
        ad, bd = T.to_dev(a), T.to_dev(b)
        r = cuda.zeros(n + 1, dtype=cuda.int32, device="cuda")
        L = qla.lib()
        for name, code in (("QLA_I_veq_I_lshift_I", 9), ("QLA_I_veq_I_rshift_I", 10), ("QLA_I_veq_I_mod_I", 5)):
            f = getattr(L, name)
            f.restype = None
            f(ctypes.c_void_p(r.data_ptr() + 4 * off), ctypes.c_void_p(ad.data_ptr() + 4 * off),
              ctypes.c_void_p(bd.data_ptr() + 4 * off), ctypes.c_int(n))
            want = np.zeros(n, np.int32)
            T.oracle().ora_int(code, 0, T.ptr(want), T.ptr(np.ascontiguousarray(a[off:off + n])),
                               T.ptr(np.ascontiguousarray(b[off:off + n])), None, 0, ctypes.c_long(n),
                               None, None, None, None)
            assert np.array_equal(T.to_host(r)[off:off + n], want), (name, off)
