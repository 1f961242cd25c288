"""Index-stream validation (qlagpu_check_index) and NVTX tracing of the
entry points, through the C-ABI."""
import os
import subprocess
import sys

import numpy as np
import pytest

import qla_testlib as T

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def test_check_index_accepts_a_neighbour_table_and_reports_bad_entries(qla, cuda):
    dims = [8, 8, 8, 16]
    n = int(np.prod(dims))
    idx = cuda.empty(n, dtype=cuda.int32, device="cuda")
    qla.shift_index(idx, dims, 2, -1)
    assert qla.check_index(idx, n, n) == (0, -1)
    # bad entries: one past the end, negative, far out; only the scan reads them
    bad = idx.clone()
    bad[5000] = n
    bad[70] = -3
    bad[n - 1] = 1 << 30
    qla.clear_error()
    rc, first = qla.check_index(bad, n, n)
    code, msg = qla.last_error()
    assert rc == 4 and first == 70 and code == 4, (rc, first, code, msg)
    assert "3 entries" in msg and "position 70" in msg and "-3" in msg, msg
    qla.clear_error()
    # a shorter source: entries >= nsrc are bad
    rc, first = qla.check_index(idx, n, n // 2)
    assert rc == 4 and first == int(np.nonzero(T.to_host(idx) >= n // 2)[0][0])
    qla.clear_error()
    # nothing to scan
    assert qla.check_index(idx, 0, 0) == (0, -1)
    assert qla.device_error() == 0


def test_nvtx_ranges_when_enabled(tmp_path):
    """With QLA_B200_NVTX=1 every entry point opens and closes an NVTX range;
    results are unchanged (checked in a fresh process, which reads the
    variable once)."""
    code = r"""
import sys, numpy as np
sys.path.insert(0, REPO); sys.path.insert(0, HERE)
import torch, qla_b200 as qla, qla_testlib as T
rng = np.random.default_rng(5)
n = 1000
a, b = T.haar_su3(rng, n), T.gaussian_field(rng, n, 3)
r = torch.empty((n, 6), dtype=torch.float32, device="cuda")
qla.F3.V_veq_M_times_V(r, T.to_dev(a), T.to_dev(b), n)
want = T.ora_lmult(np.zeros((n, 6), np.float32), a, b, n, 1, "eq")
assert T.bits_equal(T.to_host(r), want)
print("ok")
""".replace("REPO", repr(REPO)).replace("HERE", repr(HERE))
    env = dict(os.environ, QLA_B200_NVTX="1")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip().endswith("ok"), out.stderr[-2000:]
