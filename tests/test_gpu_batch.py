"""Batched uneven-volume execution (config 4 shape): 64 F3 fields with
independent lattice extents, each running r = u * u2[nbr] (QLA_F3_M_eq_M_times_xM,
neighbour gather) then w = r * v (QLA_F3_V_veq_M_times_V) in one persistent
launch.  Results must be bit-identical to the per-field calls (and to the
oracle), including partial tiles and unaligned fields, and when the launch
is replayed from a captured CUDA graph."""
import numpy as np
import pytest

import qla_testlib as T

pytestmark = pytest.mark.gpu


def _fields(cuda, rng, extents_choices, nfields, unaligned=()):
    fields, host = [], []
    for f in range(nfields):
        dims = [int(x) for x in rng.choice(extents_choices, 4)]
        n = int(np.prod(dims))
        off = 1 if f in unaligned else 0
        u = T.haar_su3(rng, n + off, np.float32)
        u2 = T.haar_su3(rng, n, np.float32)
        v = T.gaussian_field(rng, n + off, 3, np.float32)
        nbr = T.shift_index(dims, int(rng.integers(0, 4)), int(rng.choice([1, -1])))
        ud, u2d, vd = T.to_dev(u), T.to_dev(u2), T.to_dev(v)
        rd = cuda.zeros((n + off, 18), dtype=cuda.float32, device="cuda")
        wd = cuda.zeros((n + off, 6), dtype=cuda.float32, device="cuda")
        nd = T.to_dev(nbr)
        fields.append(dict(r=rd.data_ptr() + 72 * off, u=ud.data_ptr() + 72 * off, u2=u2d, nbr=nd,
                           w=wd.data_ptr() + 24 * off, v=vd.data_ptr() + 24 * off, n=n))
        host.append(dict(u=u[off:], u2=u2, v=v[off:], nbr=nbr, n=n, rd=rd, wd=wd, ud=ud, vd=vd, off=off))
    return fields, host


def _check_oracle(host, f):
    h = host[f]
    n = h["n"]
    r = np.zeros((n, 18), np.float32)
    T.ora_lmult(r, h["u"], h["u2"], n, 3, "eq", idx_b=h["nbr"])
    w = np.zeros((n, 6), np.float32)
    T.ora_lmult(w, r, h["v"], n, 1, "eq")
    off = h["off"]
    assert T.bits_equal(T.to_host(h["rd"])[off:], r), f
    assert T.bits_equal(T.to_host(h["wd"])[off:], w), f


def test_batch_small_partial_tiles_and_unaligned(qla, cuda):
    rng = np.random.default_rng(41)
    fields, host = _fields(cuda, rng, [2, 3, 4, 6], 64, unaligned=(5, 17))
    plan = qla.BatchPlan(fields)
    plan.run()
    for f in range(64):
        _check_oracle(host, f)
    plan.close()


def test_batch_config4_matches_separate_calls_and_graph_replay(qla, cuda):
    rng = np.random.default_rng(42)
    fields, host = _fields(cuda, rng, [8, 12, 16, 20, 24, 32], 64)
    plan = qla.BatchPlan(fields)
    plan.run()
    cuda.cuda.synchronize()
    got_r = [T.to_host(h["rd"]).copy() for h in host]
    got_w = [T.to_host(h["wd"]).copy() for h in host]
    # the same work as 2 x 64 separate QLA calls
    for f, h in enumerate(host):
        n = h["n"]
        r2 = cuda.empty((n, 18), dtype=cuda.float32, device="cuda")
        w2 = cuda.empty((n, 6), dtype=cuda.float32, device="cuda")
        qla.F3.M_eq_M_times_xM(r2, h["ud"], fields[f]["u2"], fields[f]["nbr"], n)
        qla.F3.V_veq_M_times_V(w2, r2, h["vd"], n)
        assert T.bits_equal(got_r[f], T.to_host(r2)), f
        assert T.bits_equal(got_w[f], T.to_host(w2)), f
    _check_oracle(host, 0)
    # replay from a captured CUDA graph
    for h in host:
        h["rd"].zero_()
        h["wd"].zero_()
    g = cuda.cuda.CUDAGraph()
    s = cuda.cuda.Stream()
    with cuda.cuda.stream(s):
        qla.set_stream(s)
        with cuda.cuda.graph(g, stream=s):
            plan.run()
    qla.set_stream(None)
    g.replay()
    g.replay()
    cuda.cuda.synchronize()
    for f, h in enumerate(host):
        assert T.bits_equal(T.to_host(h["rd"]), got_r[f]), f
        assert T.bits_equal(T.to_host(h["wd"]), got_w[f]), f
    del g
    plan.close()
    assert qla.device_error() == 0
