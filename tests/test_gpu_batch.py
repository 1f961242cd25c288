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


# ---------------------------------------------------------------------------
# per-field programs (qlagpu_F3_batch_plan_program): mixed sequences over
# fields of uneven volume in one persistent launch, each field bit-identical
# to the separate QLA_F3 calls its steps stand for

def _dev(cuda, host, off_bytes):
    """device copy of `host` (rows of records) whose first record starts
    off_bytes past a 16-B boundary; returns (address, tensor)"""
    rec = host.shape[1]
    t = cuda.zeros((host.shape[0] + 1, rec), dtype=cuda.float32, device="cuda")
    flat = t.view(-1)
    k = off_bytes // 4
    flat[k:k + host.size].copy_(cuda.from_numpy(host.reshape(-1)).cuda())
    return t.data_ptr() + off_bytes, t


def _read(cuda, t, off_bytes, n, rec):
    k = off_bytes // 4
    return t.view(-1)[k:k + n * rec].reshape(n, rec).cpu().numpy()


def _seq_config4(qla, cuda, rng, n, dims, off):
    u, u2, v = T.haar_su3(rng, n, np.float32), T.haar_su3(rng, n, np.float32), T.gaussian_field(rng, n, 3)
    nbr = T.to_dev(T.shift_index(dims, int(rng.integers(0, 4)), int(rng.choice([1, -1]))))
    (ua, ut), (u2a, u2t), (va, vt) = _dev(cuda, u, off), _dev(cuda, u2, off), _dev(cuda, v, off)
    (ra, rt), (wa, wt) = _dev(cuda, np.zeros((n, 18), np.float32), off), _dev(cuda, np.zeros((n, 6), np.float32), off)
    prog = {"n": n, "streams": [dict(base=ua, kind="M", role="in"), dict(base=u2a, index=nbr, kind="M", role="in"),
                                dict(base=va, kind="V", role="in"), dict(base=ra, kind="M", role="out"),
                                dict(base=wa, kind="V", role="out")],
            "steps": [dict(op="lmult", a=0, b=1, dst=qla.REG0, store=3),
                      dict(op="lmult", a=qla.REG0, b=2, dst=qla.REG1, store=4)]}
    keep = (ut, u2t, vt, rt, wt, nbr)

    def reference():
        r2 = cuda.empty((n, 18), dtype=cuda.float32, device="cuda")
        w2 = cuda.empty((n, 6), dtype=cuda.float32, device="cuda")
        qla.F3.M_eq_M_times_xM(r2, ua, u2a, nbr, n)
        qla.F3.V_veq_M_times_V(w2, r2, va, n)
        return [(_read(cuda, rt, off, n, 18), T.to_host(r2)), (_read(cuda, wt, off, n, 6), T.to_host(w2))]
    return prog, keep, reference, [(rt, 18), (wt, 6)]


def _seq_hop(qla, cuda, rng, n, dims, off):
    """one Wilson hop direction: out += sprecon(U spproj(D[x + mu]))"""
    mu, sg = int(rng.integers(0, 4)), int(rng.choice([1, -1]))
    u, d, o = T.haar_su3(rng, n, np.float32), T.gaussian_field(rng, n, 12), T.gaussian_field(rng, n, 12)
    nbr = T.to_dev(T.shift_index(dims, mu, sg))
    (ua, ut), (da, dt), (oa, ot) = _dev(cuda, u, off), _dev(cuda, d, off), _dev(cuda, o, off)
    prog = {"n": n, "streams": [dict(base=ua, kind="M", role="in"), dict(base=da, index=nbr, kind="D", role="in"),
                                dict(base=oa, kind="D", role="inout")],
            "steps": [dict(op="spproj", a=1, dst=qla.REG0, mu=mu, sign=sg),
                      dict(op="lmult", a=0, b=qla.REG0, dst=qla.REG1),
                      dict(op="sprecon", eqop="peq", a=qla.REG1, dst=qla.REG0, store=2, mu=mu, sign=sg)]}
    keep = (ut, dt, ot, nbr)

    def reference():
        h = cuda.empty((n, 12), dtype=cuda.float32, device="cuda")
        h2 = cuda.empty_like(h)
        out = T.to_dev(o)
        qla.F3.H_veq_spproj_D(h, da, mu, sg, n)
        qla.F3.H_eq_M_times_xH(h2, ua, h, nbr, n)
        qla.F3.D_vpeq_sprecon_H(out, h2, mu, sg, n)
        return [(_read(cuda, ot, off, n, 24), T.to_host(out))]
    return prog, keep, reference, [(ot, 24)]


def _seq_axpy_adj(qla, cuda, rng, n, dims, off):
    """y += r x (QLA_F3_D_vpeq_r_times_D), then w = U^+ y (QLA_F3_D_veq_Ma_times_D)"""
    r = float(np.float32(rng.uniform(-1, 1)))
    u, x, y = T.haar_su3(rng, n, np.float32), T.gaussian_field(rng, n, 12), T.gaussian_field(rng, n, 12)
    (ua, ut), (xa, xt), (ya, yt) = _dev(cuda, u, off), _dev(cuda, x, off), _dev(cuda, y, off)
    wa, wt = _dev(cuda, np.zeros((n, 24), np.float32), off)
    prog = {"n": n, "streams": [dict(base=ua, kind="M", role="in"), dict(base=xa, kind="D", role="in"),
                                dict(base=ya, kind="D", role="inout"), dict(base=wa, kind="D", role="out")],
            "steps": [dict(op="rtimes", eqop="peq", a=1, dst=qla.REG0, store=2, r=r),
                      dict(op="lmult", a=0, b=qla.REG0, adja=1, dst=qla.REG1, store=3)]}
    keep = (ut, xt, yt, wt)

    def reference():
        yy = T.to_dev(y)
        w2 = cuda.empty((n, 24), dtype=cuda.float32, device="cuda")
        qla.F3.D_vpeq_r_times_D(yy, r, xa, n)
        qla.F3.D_veq_Ma_times_D(w2, ua, yy, n)
        return [(_read(cuda, yt, off, n, 24), T.to_host(yy)), (_read(cuda, wt, off, n, 24), T.to_host(w2))]
    return prog, keep, reference, [(yt, 24), (wt, 24)]


def _seq_mm_adj_copy(qla, cuda, rng, n, dims, off):
    """R = U U2^+ (QLA_F3_M_veq_M_times_Ma), Q -= R (QLA_F3_M_vmeq_M)"""
    u, u2, q = T.haar_su3(rng, n, np.float32), T.gaussian_field(rng, n, 9), T.gaussian_field(rng, n, 9)
    (ua, ut), (u2a, u2t), (qa, qt) = _dev(cuda, u, off), _dev(cuda, u2, off), _dev(cuda, q, off)
    ra, rt = _dev(cuda, np.zeros((n, 18), np.float32), off)
    prog = {"n": n, "streams": [dict(base=ua, kind="M", role="in"), dict(base=u2a, kind="M", role="in"),
                                dict(base=ra, kind="M", role="out"), dict(base=qa, kind="M", role="inout")],
            "steps": [dict(op="lmult", a=0, b=1, adjb=1, dst=qla.REG0, store=2),
                      dict(op="copy", eqop="meq", a=qla.REG0, dst=qla.REG1, store=3)]}
    keep = (ut, u2t, qt, rt)

    def reference():
        r2 = cuda.empty((n, 18), dtype=cuda.float32, device="cuda")
        qq = T.to_dev(q)
        qla.F3.M_veq_M_times_Ma(r2, ua, u2a, n)
        qla.F3.M_vmeq_M(qq, r2, n)
        return [(_read(cuda, rt, off, n, 18), T.to_host(r2)), (_read(cuda, qt, off, n, 18), T.to_host(qq))]
    return prog, keep, reference, [(rt, 18), (qt, 18)]


SEQUENCES = [_seq_config4, _seq_hop, _seq_axpy_adj, _seq_mm_adj_copy]


def _mixed(qla, cuda, rng, nfields, choices, unaligned=()):
    fields = []
    for f in range(nfields):
        dims = [int(x) for x in rng.choice(choices, 4)]
        n = int(np.prod(dims))
        fields.append(SEQUENCES[f % len(SEQUENCES)](qla, cuda, rng, n, dims, 8 if f in unaligned else 0))
    return fields


@pytest.mark.parametrize("choices,nfields,unaligned", [([2, 3, 4, 6], 48, (5, 6, 17, 31)),
                                                      ([8, 12, 16, 20], 16, ())])
def test_batch_program_mixed_sequences_match_separate_calls(qla, cuda, choices, nfields, unaligned):
    rng = np.random.default_rng(43 + nfields)
    fields = _mixed(qla, cuda, rng, nfields, choices, unaligned)
    plan = qla.BatchProgramPlan([f[0] for f in fields])
    plan.run()
    cuda.cuda.synchronize()
    for k, (_, _, reference, _) in enumerate(fields):
        for got, want in reference():   # the reference starts from the INOUT streams' initial values
            assert T.bits_equal(got, want), (k, SEQUENCES[k % len(SEQUENCES)].__name__)
    plan.close()
    assert qla.device_error() == 0


def test_batch_program_graph_replay_and_reruns(qla, cuda):
    """OUT-only programs give the same bits on every replay; the replayed
    launch equals the eager one."""
    rng = np.random.default_rng(47)
    fields = []
    for f in range(12):
        dims = [int(x) for x in rng.choice([4, 6, 8, 12], 4)]
        n = int(np.prod(dims))
        seq = (_seq_config4, _seq_mm_adj_copy)[f % 2]
        fields.append(seq(qla, cuda, rng, n, dims, 0))
    # drop the INOUT step of the M M^+ sequence so that reruns are idempotent
    progs = []
    for p, _, _, _ in fields:
        if len(p["streams"]) == 4 and p["streams"][3]["role"] == "inout":
            p = dict(p, streams=p["streams"][:3], steps=p["steps"][:1])
        progs.append(p)
    plan = qla.BatchProgramPlan(progs)
    plan.run()
    cuda.cuda.synchronize()
    first = [[_read(cuda, t, 0, f[0]["n"], rec).copy() for t, rec in f[3][:1]] for f in fields]
    for f in fields:
        for t, _ in f[3][:1]:
            t.zero_()
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
    for k, f in enumerate(fields):
        for (t, rec), want in zip(f[3][:1], first[k]):
            assert T.bits_equal(_read(cuda, t, 0, f[0]["n"], rec), want), k
    del g
    plan.close()
    assert qla.device_error() == 0


def test_batch_program_checks_gather_indices(qla, cuda):
    """With nsrc set, an index outside [0, nsrc) raises QLA_DEVERR_BAD_INDEX
    and that site reads zeros; every other site is unaffected.  (The kernel
    checks before it dereferences, so no out-of-range address is read.)"""
    rng = np.random.default_rng(48)
    n = 4096 + 100  # full tiles and a partial one
    u, u2 = T.haar_su3(rng, n, np.float32), T.haar_su3(rng, n, np.float32)
    idx = rng.permutation(n).astype(np.int32)
    bad = np.array([3, 700, 4150])
    idx[bad] = np.array([n, -1, n + 12345], np.int32)
    ud, u2d, rd = T.to_dev(u), T.to_dev(u2), cuda.full((n, 18), 7.0, dtype=cuda.float32, device="cuda")
    prog = {"n": n, "streams": [dict(base=ud, kind="M", role="in"),
                                dict(base=u2d, index=T.to_dev(idx), nsrc=n, kind="M", role="in"),
                                dict(base=rd, kind="M", role="out")],
            "steps": [dict(op="lmult", a=0, b=1, dst=qla.REG0, store=2)]}
    qla.device_error()  # clear the device error word ...
    qla.clear_error()   # ... and the sticky status
    plan = qla.BatchProgramPlan([prog])
    plan.run()
    cuda.cuda.synchronize()
    assert qla.device_error() & 4
    got = T.to_host(rd)
    good = np.setdiff1d(np.arange(n), bad)
    want = np.zeros((n, 18), np.float32)
    T.ora_lmult(want, u, u2, n, 3, "eq", idx_b=np.where(np.isin(np.arange(n), bad), 0, idx))
    assert T.bits_equal(got[good], want[good])
    assert np.all(got[bad] == 0.0)
    plan.close()
    qla.clear_error()
