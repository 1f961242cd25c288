"""GPU parity of the global reductions (norm2, dot, re_dot) against the
oracle, through the C-ABI.

Reference semantics (lib/perl/build_qla.pl:2089-2360): a sequential sum in
double.  The GPU forms each product exactly in double and accumulates in
double-double, so it is *more* accurate than the reference.  Tolerances,
stated per comparison:
  * against the extended-precision oracle (double-double):  rel <= 1e-12
    (observed ~1e-16);
  * against the reference-order oracle: the reference's own rounding, i.e.
    rel <= 1e-6 when it rounds each F3 term to float, rel <= 1e-12 for D3;
  * F3 functions return float: within 1 ulp of the correctly rounded value.
"""
import ctypes
import itertools

import numpy as np
import pytest

import qla_testlib as T

pytestmark = pytest.mark.gpu

REC_B = {"F3": 8, "D3": 16, "DF3": 8}


def _rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("DF3", np.float32), ("D3", np.float64)])
@pytest.mark.parametrize("t", ["V", "H", "D", "M"])
def test_norm2_dot_variants(qla, cuda, pc, dt, t):
    rng = np.random.default_rng(3 + ord(t))
    n, ns = 3001, 3100
    nc = T.NCPLX3[t]
    a_src = T.gaussian_field(rng, ns, nc, dt)
    b_src = T.gaussian_field(rng, ns, nc, dt)
    ia = rng.integers(0, ns, n).astype(np.int32)
    ib = rng.integers(0, ns, n).astype(np.int32)
    gang = rng.permutation(n).astype(np.int32)
    ad, bd = T.to_dev(a_src), T.to_dev(b_src)
    pa = T.ptr_array(ad, ia, REC_B[pc] * nc)
    pb = T.ptr_array(bd, ib, REC_B[pc] * nc)
    ns_ = getattr(qla, pc)
    outdt = cuda.float32 if pc == "F3" else cuda.float64
    for var, p1, p2 in itertools.product(["v", "x"], [0, 1], [0, 1]):
        extra = [T.to_dev(gang)] if var == "x" else []
        g = gang if var == "x" else None
        xa = ia if p1 else None
        xb = ib if p2 else None
        sa = ("p" if p1 else "") + t
        sb = ("p" if p2 else "") + t
        if not p2:
            # norm2, host output (synchronous) and device output (asynchronous)
            got_h = getattr(ns_, f"r_{var}eq_norm2_{sa}")(None, pa if p1 else ad, *extra, n)
            out = cuda.zeros(1, dtype=outdt, device="cuda")
            getattr(ns_, f"r_{var}eq_norm2_{sa}")(out, pa if p1 else ad, *extra, n)
            got_d = float(out.cpu()[0])
            exact = T.ora_norm2(a_src, n, nc, exact=True, idx_a=xa, gang=g)
            refo = T.ora_norm2(a_src, n, nc, exact=False, idx_a=xa, gang=g)
            assert got_h == got_d
            if pc == "F3":
                assert got_h == float(np.float32(exact)) or _rel(got_h, exact) <= 6e-8, (var, p1)
                assert _rel(got_h, refo) <= 1e-6
            else:
                assert _rel(got_h, exact) <= 1e-12, (var, p1, got_h, exact)
                assert _rel(got_h, refo) <= (1e-6 if pc == "DF3" else 1e-12)
        # complex dot
        got = getattr(ns_, f"c_{var}eq_{sa}_dot_{sb}")(None, pa if p1 else ad, pb if p2 else bd, *extra, n)
        exact = T.ora_dot(a_src, b_src, n, nc, exact=True, idx_a=xa, idx_b=xb, gang=g)
        refo = T.ora_dot(a_src, b_src, n, nc, exact=False, idx_a=xa, idx_b=xb, gang=g)
        scale = max(abs(exact), 1.0)
        tol = 6e-8 if pc == "F3" else 1e-12
        assert abs(got - exact) <= tol * scale * 2, (var, p1, p2, got, exact)
        assert abs(got - refo) <= (1e-6 if pc == "F3" else 1e-12) * scale * 2
        gr = getattr(ns_, f"r_{var}eq_re_{sa}_dot_{sb}")(None, pa if p1 else ad, pb if p2 else bd, *extra, n)
        assert abs(gr - exact.real) <= tol * scale * 2


@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64)])
def test_reduction_edge_sizes(qla, pc, dt):
    """n <= 0 stores a zero sum (the reference loops zero times); tiny and
    tile-boundary sizes; repeated calls reuse the scratch (ticket counter)."""
    rng = np.random.default_rng(9)
    ns_ = getattr(qla, pc)
    a = T.gaussian_field(rng, 5000, 12, dt)
    ad = T.to_dev(a)
    assert ns_.r_veq_norm2_D(None, ad, 0) == 0.0
    assert ns_.c_veq_D_dot_D(None, ad, ad, -3) == 0.0
    for n in (1, 2, 31, 64, 65, 128, 255, 256, 257, 4095, 5000):
        for _ in range(2):
            got = ns_.r_veq_norm2_D(None, ad, n)
            exact = T.ora_norm2(a, n, 12, exact=True)
            assert _rel(got, exact) <= (6e-8 if pc == "F3" else 1e-12), n


def test_reduction_determinism(qla):
    rng = np.random.default_rng(1)
    a = T.gaussian_field(rng, 200003, 12, np.float32)
    ad = T.to_dev(a)
    vals = {qla.DF3.r_veq_norm2_D(None, ad, 200003) for _ in range(5)}
    assert len(vals) == 1


def test_full_size_cg_chain_reductions(qla, cuda):
    """48^3x96 DiracFermion fields (10,616,832 sites): the FP32-site /
    FP64-reduction chain agrees with the extended-precision oracle to
    <= 1e-12 relative, and the F3 axpy is bit-exact (checked by a checksum of
    the full output against the oracle's)."""
    n = 48 * 48 * 48 * 96
    g = cuda.Generator(device="cuda")
    g.manual_seed(1234)
    x = cuda.randn(n, 24, device="cuda", dtype=cuda.float32, generator=g)
    p = cuda.randn(n, 24, device="cuda", dtype=cuda.float32, generator=g)
    xh, ph = x.cpu().numpy(), p.cpu().numpy()
    a = np.float32(0.37)
    qla.F3.D_vpeq_r_times_D(x, float(a), p, n)
    nrm = qla.DF3.r_veq_norm2_D(None, x, n)
    dot = qla.DF3.c_veq_D_dot_D(None, x, p, n)
    want_x = xh.copy()
    T.ora_rtimes(want_x, float(a), ph, n, 12, "peq")
    assert T.bits_equal(x.cpu().numpy(), want_x)
    e_n = T.ora_norm2(want_x, n, 12, exact=True)
    e_d = T.ora_dot(want_x, ph, n, 12, exact=True)
    assert _rel(nrm, e_n) <= 1e-12
    assert abs(dot - e_d) <= 1e-12 * abs(e_d)


@pytest.mark.parametrize("rp,dt", [("D3", np.float64), ("DF3", np.float32), ("F3", np.float32)])
def test_reductions_on_large_fields_match_the_direct_path(qla, cuda, rp, dt):
    """Fields of 2^24 complex numbers run the pipelined kernel with many tiles
    per block, so every shared-memory stage is refilled many times.  Each of
    three repeated calls must equal the direct path's result bit for bit (the
    same per-site terms, both summed in double-double), and match the
    long-double sum of the data.  A stage refilled before its consumers had
    finished reading it showed up here first, as run-to-run differences of
    the D3 DiracFermion norm2 at the 1e-7 level."""
    import math
    g = cuda.Generator(device="cuda")
    g.manual_seed(11)
    V = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    L = qla.lib()
    out = cuda.zeros(4, dtype=cuda.float32 if rp == "F3" else cuda.float64, device="cuda")
    for t in ("V", "H", "D", "M"):
        nc = T.NCPLX3[t]
        n = (1 << 24) // nc
        x = cuda.randn(n, 2 * nc, device="cuda", dtype=cuda.float32 if dt == np.float32 else cuda.float64,
                       generator=g)
        y = cuda.randn_like(x)
        gang = cuda.arange(n, dtype=cuda.int32, device="cuda")
        getattr(L, f"QLA_{rp}_r_xeq_norm2_{t}")(V(out), V(x), V(gang), n)
        getattr(L, f"QLA_{rp}_c_xeq_{t}_dot_{t}")(V(out[1:]), V(x), V(y), V(gang), n)
        ref = out[:3].cpu().numpy().copy()
        for _ in range(3):
            getattr(L, f"QLA_{rp}_r_veq_norm2_{t}")(V(out), V(x), n)
            getattr(L, f"QLA_{rp}_c_veq_{t}_dot_{t}")(V(out[1:]), V(x), V(y), n)
            got = out[:3].cpu().numpy()
            assert np.array_equal(got, ref), (t, got, ref)
        qla.check("large reductions")
        xs = x.cpu().numpy().astype(np.longdouble)
        exact = math.fsum((xs * xs).sum(axis=1).astype(np.float64))
        tol = 6e-8 if rp == "F3" else 1e-12
        assert abs(float(ref[0]) - exact) <= tol * exact, (t, ref[0], exact)
        del x, y, gang, xs
