"""The allocation-free norm2 entry point, qlagpu_DF3_r_veq_norm2_D_noalloc,
called through the C-ABI.

It exists for host programs that cannot call cudaMalloc while they run: a
lattice code whose own pool allocator reserved the device memory up front, or
one working under a hard memory budget.  The regular reductions allocate their
scratch on first use; this entry point keeps its scratch in a static device
array instead.  Its results must agree with the regular entry point
QLA_DF3_r_veq_norm2_D to the reductions' stated tolerance (rel <= 1e-12; the
two use different grids, hence different summation orders), on two calls in a
row (the static array keeps the previous call's contents).

The first test runs in a fresh child process with tests/cuda_alloc_counter.c
preloaded, which counts the CUDA runtime's allocation and release calls: the
entry point's first call on the device (the set-up) and the calls after it
make none, and the device's free memory does not change across them.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process."""
import ctypes
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
MAX_SITES = 65536 * 256
TMA_BLOCK, DIRECT_BLOCK, FOLD_BLOCK = 256 + 32, 256, 1


def _entry(qla):
    f = qla.lib().qlagpu_DF3_r_veq_norm2_D_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    return f


def _rel(a, b):
    return abs(a - b) / abs(b)


_CHILD = r"""
import ctypes, json, sys
import numpy as np
import torch
sys.path.insert(0, REPO)
torch.cuda.init()
counter = ctypes.CDLL(COUNTER)
counter.qla_test_alloc_calls.restype = ctypes.c_long
blocks = (ctypes.c_uint * 256)()
def launches():
    k = counter.qla_test_launches(blocks, 256)
    return [int(blocks[i]) for i in range(min(k, 256))]
n = 1_000_003
x = torch.randn(n, 24, device="cuda", dtype=torch.float32)
ys = torch.randn(1000, 24, device="cuda", dtype=torch.float32)
dev_out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
want = float((x.double() ** 2).sum())
torch.cuda.synchronize()
import qla_b200
L = qla_b200.lib()
f = L.qlagpu_DF3_r_veq_norm2_D_noalloc
f.restype = ctypes.c_int
f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
out = {}
a0 = counter.qla_test_alloc_calls()
r = ctypes.c_double(-1.0)
counter.qla_test_reset_launches()
out["rc_first"] = f(ctypes.addressof(r), x.data_ptr(), n)   # first call on the device: the set-up
out["launch_first"] = launches()
out["rel_first"] = abs(r.value - want) / want
# a start 8 B past a 16-B boundary (half a complex number into a record):
# bulk copies need 16-B alignment, so this takes the direct kernel
ysh = ys.cpu().numpy().reshape(-1)[2:2 + 999 * 24].astype(np.float64)
want_y = float((ysh ** 2).sum())
rels = []
out["rcs"] = []
counter.qla_test_reset_launches()
out["rcs"].append(f(ctypes.addressof(r), ys.data_ptr() + 8, 999))
out["launch_unaligned"] = launches()
rels.append(abs(r.value - want_y) / want_y)
out["allocs_first"] = counter.qla_test_alloc_calls() - a0
# every kernel has run once (its code is loaded); the device's free memory
# must not change across further calls
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info()[0]
a1 = counter.qla_test_alloc_calls()
for _ in range(2):
    out["rcs"].append(f(ctypes.addressof(r), x.data_ptr(), n))
    rels.append(abs(r.value - want) / want)
    out["rcs"].append(f(dev_out.data_ptr(), x.data_ptr(), n))
    torch.cuda.synchronize()
    rels.append(abs(float(dev_out.cpu()[0]) - want) / want)
    out["rcs"].append(f(ctypes.addressof(r), ys.data_ptr() + 8, 999))
    rels.append(abs(r.value - want_y) / want_y)
out["allocs_after"] = counter.qla_test_alloc_calls() - a1
torch.cuda.synchronize()
out["free_delta"] = torch.cuda.mem_get_info()[0] - free0
out["rels"] = rels
out["device_error"] = int(L.qlagpu_device_error(0))
print("RESULT " + json.dumps(out))
"""


def test_noalloc_first_call_allocates_nothing_in_a_fresh_process(tmp_path):
    so = os.path.join(str(tmp_path), "libcuda_alloc_counter.so")
    subprocess.check_call(["gcc", "-O2", "-shared", "-fPIC", "-o", so,
                           os.path.join(HERE, "cuda_alloc_counter.c"), "-ldl"])
    env = dict(os.environ, LD_PRELOAD=so)
    code = _CHILD.replace("REPO", repr(REPO)).replace("COUNTER", repr(so))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-4000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("RESULT ")]
    assert line, r.stdout[-2000:] + r.stderr[-2000:]
    out = json.loads(line[-1][len("RESULT "):])
    assert out["rc_first"] == 0 and all(rc == 0 for rc in out["rcs"]), out
    assert out["allocs_first"] == 0, out      # the first call's set-up allocates nothing
    assert out["allocs_after"] == 0, out      # neither do the calls after it
    assert out["free_delta"] == 0, out        # the device's free memory is unchanged
    assert out["launch_first"] == [TMA_BLOCK, FOLD_BLOCK], out
    assert out["launch_unaligned"] == [DIRECT_BLOCK, FOLD_BLOCK], out
    assert out["rel_first"] <= 1e-12 and max(out["rels"]) <= 1e-12, out
    assert out["device_error"] == 0, out


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
    # small sizes, whole records past the start (16-B aligned: pipelined
    # kernel) and a start half a complex number into a record (8-B aligned:
    # direct kernel), each against the regular entry point at the same address
    for n, off_bytes in ((1, 0), (255, 0), (256, 0), (257, 0), (999, 96), (999, 8), (300, 8)):
        out = ctypes.c_double()
        rc = f(ctypes.addressof(out), x.data_ptr() + off_bytes, n)
        assert rc == 0
        want = qla.DF3.r_veq_norm2_D(None, x.data_ptr() + off_bytes, n)
        assert _rel(out.value, want) <= 1e-12, (n, off_bytes)
    out = ctypes.c_double(5.0)
    assert f(ctypes.addressof(out), x.data_ptr(), 0) == 0 and out.value == 0.0
    # beyond the static scratch: rejected before any device access
    qla.clear_error()
    assert f(ctypes.addressof(out), x.data_ptr(), MAX_SITES + 1) == 4
    code, msg = qla.last_error()
    assert code == 4 and "16777216" in msg
    qla.clear_error()
    assert qla.device_error() == 0
