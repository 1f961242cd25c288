"""Failure detection without a GPU fault: every pipeline wait in the kernels
is time-bounded.  A kernel made to wait on a barrier phase that nothing
completes must give up after its limit, report the timeout through the
device error word, and leave the context usable (further calls succeed and
stay bit-exact)."""
import numpy as np
import pytest

import qla_testlib as T

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_survives(qla):
    L = qla.lib()
    assert L.qlagpu_selftest_wait_timeout(2000) == 1      # 2 ms limit
    assert qla.device_error() == 0                         # bit consumed by the self-test
    rng = np.random.default_rng(3)
    n = 4096
    a = T.haar_su3(rng, n, np.float32)
    b = T.gaussian_field(rng, n, 3, np.float32)
    r = T.to_dev(np.zeros((n, 6), np.float32))
    qla.F3.V_veq_M_times_V(r, T.to_dev(a), T.to_dev(b), n)
    want = np.zeros((n, 6), np.float32)
    T.ora_lmult(want, a, b, n, 1, "eq")
    assert T.bits_equal(T.to_host(r), want)


def test_host_side_argument_errors(qla):
    L = qla.lib()
    qla.clear_error()
    assert L.qlagpu_selftest_wait_timeout(0) == -1
    assert qla.last_error()[0] == 4
    qla.clear_error()
    L.qlagpu_shift_index(None, 4, None, 0, 1)
    assert qla.last_error()[0] == 1
    qla.clear_error()
