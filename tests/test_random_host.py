"""CPU check of the library's host random-number functions on one state in
host memory (QLA_seed_random, QLA_random, QLA_gaussian with and without
QLA_use_milc_gaussian): bit-identical values and states to the oracle, which
is pinned to the reference's lib/random (tests/test_oracle_pin.py).  These
are the reference's host API; the field fills run on the device."""
import ctypes
import os

import numpy as np
import pytest

import qla_testlib as T

LIB = os.path.join(T.REPO, "qla_b200", "lib", "libqla_b200.so")


@pytest.mark.skipif(not os.path.exists(LIB), reason="libqla_b200.so not built")
@pytest.mark.parametrize("milc", [0, 1])
def test_host_generator_matches_oracle(milc):
    L = ctypes.CDLL(LIB)
    O = T.oracle()
    L.QLA_random.restype = ctypes.c_float
    L.QLA_gaussian.restype = ctypes.c_float
    O.ora_rng_uniform.restype = ctypes.c_float
    O.ora_rng_gaussian.restype = ctypes.c_float
    flag = ctypes.c_int.in_dll(L, "QLA_use_milc_gaussian")
    flag.value = milc
    try:
        rng = np.random.default_rng(120)
        for _ in range(30):
            seed, index = int(rng.integers(-2**31, 2**31 - 1)), int(rng.integers(0, 1 << 22))
            a = np.zeros(11, np.uint32)
            b = np.zeros(11, np.uint32)
            L.QLA_seed_random(T.ptr(a), seed, index)
            O.ora_rng_seed(T.ptr(b), seed, index)
            assert T.bits_equal(a, b)
            for j in range(200):
                if j % 4 == 0:
                    x, y = L.QLA_random(T.ptr(a)), O.ora_rng_uniform(T.ptr(b))
                else:
                    x, y = L.QLA_gaussian(T.ptr(a)), O.ora_rng_gaussian(T.ptr(b), milc)
                assert np.float32(x).tobytes() == np.float32(y).tobytes()
            assert T.bits_equal(a, b)
    finally:
        flag.value = 0
