"""GPU parity of the linear level-1 families against the oracle, through the
C-ABI (libqla_b200.so): every eqop, adjoint, pointer (`pX`), gang-index
(`x`) and per-operand index (`xX`) variant.  The kernels round every
multiply and add separately, in the reference's order, so results must be
bit-identical to the oracle (which is itself bit-identical to the reference
library, tests/test_oracle_pin.py)."""
import itertools

import numpy as np
import pytest

import qla_testlib as T

pytestmark = pytest.mark.gpu

PCS = [("F3", np.float32), ("D3", np.float64)]
REC_B = {"F3": 8, "D3": 16}  # bytes per complex


def rec_bytes(pc, t):
    return REC_B[pc] * T.NCPLX3[t]


def _perm(rng, n):
    return rng.permutation(n).astype(np.int32)


@pytest.mark.parametrize("pc,dt", PCS)
@pytest.mark.parametrize("dest", ["V", "H", "D", "M"])
def test_lmult_all_variants(qla, pc, dt, dest):
    rng = np.random.default_rng(11 + ord(dest))
    n = 1031  # not a multiple of any tile: exercises the partial tail tile
    ns = n + 17  # gather sources are larger than the destination
    ncol = T.NCOL3[dest]
    a_src = T.haar_su3(rng, ns, dt)
    b_src = T.gaussian_field(rng, ns, T.NCPLX3[dest], dt)
    r0 = T.gaussian_field(rng, n, T.NCPLX3[dest], dt)
    ia = rng.integers(0, ns, n).astype(np.int32)
    ib = rng.integers(0, ns, n).astype(np.int32)
    gang = _perm(rng, n)
    a_d, b_d = T.to_dev(a_src), T.to_dev(b_src)
    pa = T.ptr_array(a_d, ia, rec_bytes(pc, "M"))
    pb = T.ptr_array(b_d, ib, rec_bytes(pc, dest))
    ns_ = getattr(qla, pc)
    src2s = [(dest, 0), ("p" + dest, 0)] + ([("Ma", 1), ("pMa", 1)] if dest == "M" else [])
    nchecked = 0
    for var, eq, s1, (s2, adjb) in itertools.product(["v", "x"], T.EQOPS, ["M", "Ma", "pM", "pMa"], src2s):
        adja = 1 if s1.endswith("a") else 0
        p1, p2 = s1.startswith("p"), s2.startswith("p")
        r_d = T.to_dev(r0)
        args = [r_d, pa if p1 else a_d, pb if p2 else b_d]
        if var == "x":
            args.append(T.to_dev(gang))
        args.append(n)
        getattr(ns_, f"{dest}_{var}{eq}_{s1}_times_{s2}")(*args)
        got = T.to_host(r_d)
        want = r0.copy()
        T.ora_lmult(want, a_src, b_src, n, ncol, eq, adja=adja, adjb=adjb,
                    idx_a=ia if p1 else None, idx_b=ib if p2 else None,
                    gang=gang if var == "x" else None)
        assert T.bits_equal(got, want), f"{pc}_{dest}_{var}{eq}_{s1}_times_{s2}"
        nchecked += 1
    # per-operand int32 index (the neighbour-gather form)
    for eq, s1 in itertools.product(T.EQOPS, ["M", "Ma"]):
        r_d = T.to_dev(r0)
        getattr(ns_, f"{dest}_{eq}_{s1}_times_x{dest}")(r_d, a_d, b_d, T.to_dev(ib), n)
        want = r0.copy()
        T.ora_lmult(want, a_src, b_src, n, ncol, eq, adja=int(s1 == "Ma"), idx_b=ib)
        assert T.bits_equal(T.to_host(r_d), want), f"{pc}_{dest}_{eq}_{s1}_times_x{dest}"
        nchecked += 1
    assert nchecked > 64


@pytest.mark.parametrize("pc,dt", PCS)
@pytest.mark.parametrize("n", [1, 2, 63, 64, 65, 255, 256, 257, 4099, 70001])
def test_mv_sizes_and_alignment(qla, pc, dt, n):
    """Sizes around the tile boundaries, and sub-16-byte-aligned pointers that
    take the direct (non-bulk-copy) path."""
    rng = np.random.default_rng(n)
    a = T.haar_su3(rng, n + 1, dt)
    b = T.gaussian_field(rng, n + 1, 3, dt)
    r0 = T.gaussian_field(rng, n + 1, 3, dt)
    ns_ = getattr(qla, pc)
    for off in (0, 1):
        a_d, b_d, r_d = T.to_dev(a), T.to_dev(b), T.to_dev(r0)
        ao = a_d.data_ptr() + off * rec_bytes(pc, "M")
        bo = b_d.data_ptr() + off * rec_bytes(pc, "V")
        ro = r_d.data_ptr() + off * rec_bytes(pc, "V")
        ns_.V_vpeq_M_times_V(ro, ao, bo, n)
        want = r0.copy()
        T.ora_lmult(want[off:], a[off:], b[off:], n, 1, "peq")
        assert T.bits_equal(T.to_host(r_d), want), (n, off)


@pytest.mark.parametrize("pc,dt", PCS)
def test_spproj_sprecon(qla, pc, dt):
    rng = np.random.default_rng(5)
    n, ns = 777, 800
    d_src = T.gaussian_field(rng, ns, 12, dt)
    h_src = T.gaussian_field(rng, ns, 6, dt)
    h0 = T.gaussian_field(rng, n, 6, dt)
    d0 = T.gaussian_field(rng, n, 12, dt)
    ia = rng.integers(0, ns, n).astype(np.int32)
    gang = _perm(rng, n)
    dd, hd = T.to_dev(d_src), T.to_dev(h_src)
    pdd = T.ptr_array(dd, ia, rec_bytes(pc, "D"))
    phd = T.ptr_array(hd, ia, rec_bytes(pc, "H"))
    ns_ = getattr(qla, pc)
    for var, eq, p1, mu, sign in itertools.product(["v", "x"], T.EQOPS, [0, 1], range(5), [1, -1]):
        extra = [T.to_dev(gang)] if var == "x" else []
        r_d = T.to_dev(h0)
        getattr(ns_, f"H_{var}{eq}_spproj_{'p' if p1 else ''}D")(r_d, pdd if p1 else dd, mu, sign, *extra, n)
        want = h0.copy()
        T.ora_spproj(want, d_src, n, mu, sign, eq, idx_a=ia if p1 else None, gang=gang if var == "x" else None)
        assert T.bits_equal(T.to_host(r_d), want), ("spproj", var, eq, p1, mu, sign)
        r_d = T.to_dev(d0)
        getattr(ns_, f"D_{var}{eq}_sprecon_{'p' if p1 else ''}H")(r_d, phd if p1 else hd, mu, sign, *extra, n)
        want = d0.copy()
        T.ora_sprecon(want, h_src, n, mu, sign, eq, idx_a=ia if p1 else None, gang=gang if var == "x" else None)
        assert T.bits_equal(T.to_host(r_d), want), ("sprecon", var, eq, p1, mu, sign)
    # mu outside 0..4 is a no-op, as in the reference
    r_d = T.to_dev(h0)
    ns_.H_veq_spproj_D(r_d, dd, 5, 1, n)
    assert T.bits_equal(T.to_host(r_d), h0)


@pytest.mark.parametrize("pc,dt", PCS)
@pytest.mark.parametrize("t", ["V", "H", "D", "M"])
def test_rtimes_and_copy(qla, cuda, pc, dt, t):
    rng = np.random.default_rng(7)
    n, ns = 2049, 2100
    nc = T.NCPLX3[t]
    b_src = T.gaussian_field(rng, ns, nc, dt)
    r0 = T.gaussian_field(rng, n, nc, dt)
    ib = rng.integers(0, ns, n).astype(np.int32)
    gang = _perm(rng, n)
    bd = T.to_dev(b_src)
    pb = T.ptr_array(bd, ib, rec_bytes(pc, t))
    ns_ = getattr(qla, pc)
    s = float(np.array(-0.7312, dtype=dt))
    s_dev = cuda.tensor([s], dtype=cuda.float32 if dt == np.float32 else cuda.float64, device="cuda")
    for var, eq, p1, scal in itertools.product(["v", "x"], T.EQOPS, [0, 1], ["host", "dev"]):
        extra = [T.to_dev(gang)] if var == "x" else []
        r_d = T.to_dev(r0)
        getattr(ns_, f"{t}_{var}{eq}_r_times_{'p' if p1 else ''}{t}")(r_d, s if scal == "host" else s_dev,
                                                                       pb if p1 else bd, *extra, n)
        want = r0.copy()
        T.ora_rtimes(want, s, b_src, n, nc, eq, idx_b=ib if p1 else None, gang=gang if var == "x" else None)
        assert T.bits_equal(T.to_host(r_d), want), ("rtimes", var, eq, p1, scal)
        if scal == "dev":
            continue
        r_d = T.to_dev(r0)
        getattr(ns_, f"{t}_{var}{eq}_{'p' if p1 else ''}{t}")(r_d, pb if p1 else bd, *extra, n)
        got = T.to_host(r_d)
        want = r0.copy()
        sel = gang if var == "x" else np.arange(n)
        src = b_src[ib[sel]] if p1 else b_src[sel]
        if eq == "eq":
            want[sel] = src
        elif eq == "eqm":
            want[sel] = -src
        elif eq == "peq":
            want[sel] = want[sel] + src
        else:
            want[sel] = want[sel] - src
        assert T.bits_equal(got, want), ("copy", var, eq, p1)
    # per-operand index gather
    r_d = T.to_dev(r0)
    getattr(ns_, f"{t}_eq_x{t}")(r_d, bd, T.to_dev(ib), n)
    assert T.bits_equal(T.to_host(r_d), b_src[ib])


def test_shift_index_bit_exact(qla, cuda):
    for dims in ([4, 4, 4, 4], [8, 6, 4, 2], [32, 32, 32, 64], [5, 3, 7]):
        n = int(np.prod(dims))
        for mu in range(len(dims)):
            for sign in (1, -1):
                idx = cuda.empty(n, dtype=cuda.int32, device="cuda")
                qla.shift_index(idx, dims, mu, sign)
                assert np.array_equal(T.to_host(idx), T.shift_index(dims, mu, sign)), (dims, mu, sign)


@pytest.mark.parametrize("pc,dt", PCS)
def test_fused_hop_terms(qla, pc, dt):
    """D_vpeq_spproj_M_times_pD and its family (the Wilson hop terms), every
    eqop / adjoint / pointer / gang / index form and every mu, sign."""
    rng = np.random.default_rng(88)
    n, ns = 517, 560
    a = T.haar_su3(rng, ns, dt)
    d_src = T.gaussian_field(rng, ns, 12, dt)
    h_src = T.gaussian_field(rng, ns, 6, dt)
    r0 = {"H": T.gaussian_field(rng, ns, 6, dt), "D": T.gaussian_field(rng, ns, 12, dt)}
    idx = rng.integers(0, ns, ns).astype(np.int32)
    gang = rng.permutation(n).astype(np.int32)
    ad, dd, hd = T.to_dev(a), T.to_dev(d_src), T.to_dev(h_src)
    pa = T.ptr_array(ad, idx, rec_bytes(pc, "M"))
    pdd = T.ptr_array(dd, idx, rec_bytes(pc, "D"))
    phd = T.ptr_array(hd, idx, rec_bytes(pc, "H"))
    ns_ = getattr(qla, pc)
    count = 0
    for (dest, kind), eq, s1, pb, var in itertools.product(
            [("H", "spproj"), ("D", "spproj"), ("D", "sprecon")], T.EQOPS, ["M", "Ma", "pM"], [0, 1], ["v", "x"]):
        src = "D" if kind == "spproj" else "H"
        bsrc, bdev, bptr = (d_src, dd, pdd) if src == "D" else (h_src, hd, phd)
        for mu, sign in ((0, 1), (1, -1), (2, 1), (3, -1), (4, 1), (4, -1)):
            r_d = T.to_dev(r0[dest][:n])
            args = [r_d, pa if s1.startswith("p") else ad, bptr if pb else bdev, mu, sign]
            if var == "x":
                args.append(T.to_dev(gang))
            getattr(ns_, f"{dest}_{var}{eq}_{kind}_{s1}_times_{'p' if pb else ''}{src}")(*args, n)
            want = r0[dest][:n].copy()
            aa = a[idx[:n]] if s1.startswith("p") else a[:n]
            T.ora_hop(want, np.ascontiguousarray(aa), bsrc, n, mu, sign, eq, dest, kind, adja=int(s1.endswith("a")),
                      idx_b=idx if pb else None, gang=gang if var == "x" else None)
            assert T.bits_equal(T.to_host(r_d), want), (dest, kind, var, eq, s1, pb, mu, sign)
            count += 1
    # int32 neighbour-index form and the D-destination projection
    for (dest, kind), eq in itertools.product([("H", "spproj"), ("D", "spproj"), ("D", "sprecon")], T.EQOPS):
        src = "D" if kind == "spproj" else "H"
        bsrc, bdev = (d_src, dd) if src == "D" else (h_src, hd)
        r_d = T.to_dev(r0[dest][:n])
        getattr(ns_, f"{dest}_{eq}_{kind}_M_times_x{src}")(r_d, ad, bdev, T.to_dev(idx), 2, -1, n)
        want = r0[dest][:n].copy()
        T.ora_hop(want, np.ascontiguousarray(a[:n]), bsrc, n, 2, -1, eq, dest, kind, idx_b=idx)
        assert T.bits_equal(T.to_host(r_d), want), (dest, kind, eq, "xb")
    for eq, mu in itertools.product(T.EQOPS, range(5)):
        r_d = T.to_dev(r0["D"][:n])
        getattr(ns_, f"D_v{eq}_spproj_D")(r_d, dd, mu, 1, n)
        want = r0["D"][:n].copy()
        T.ora_hop(want, None, d_src, n, mu, 1, eq, "D", "spproj")
        assert T.bits_equal(T.to_host(r_d), want), ("Dspproj", eq, mu)
    assert count > 400


@pytest.mark.parametrize("pc,dt", PCS)
@pytest.mark.parametrize("nd", [1, 3, 8, 11])
def test_multi_direction_sum(qla, cuda, pc, dt, nd):
    """V_{v,x}{eqop}_n{p}M{a}_times_n{p}V: r (eqop) sum_d A_d b_d with the
    reference's per-direction rounding; nd = 11 runs in two launches;
    operand tables on the host and on the device."""
    rng = np.random.default_rng(90 + nd)
    n, ns = 1037, 1100
    ms = [T.haar_su3(rng, ns, dt) for _ in range(nd)]
    vs = [T.gaussian_field(rng, ns, 3, dt) for _ in range(nd)]
    r0 = T.gaussian_field(rng, n, 3, dt)
    ia = rng.integers(0, ns, ns).astype(np.int32)
    ib = rng.integers(0, ns, ns).astype(np.int32)
    gang = _perm(rng, n)
    md = [T.to_dev(m) for m in ms]
    vd = [T.to_dev(v) for v in vs]
    pms = [T.ptr_array(m, ia, rec_bytes(pc, "M")) for m in md]
    pvs = [T.ptr_array(v, ib, rec_bytes(pc, "V")) for v in vd]
    import ctypes
    L = qla.lib()

    def table(ts, on_dev):
        addrs = np.array([t.data_ptr() for t in ts], dtype=np.int64)
        if on_dev:
            d = T.to_dev(addrs)
            return d, d.data_ptr()
        return addrs, addrs.ctypes.data

    for var, eq, s1, s2 in itertools.product(["v", "x"], T.EQOPS, ["nM", "nMa", "npM"], ["nV", "npV"]):
        on_dev = (eq in ("peq", "eqm"))
        keep_a, a_addr = table(pms if "p" in s1 else md, on_dev)
        keep_b, b_addr = table(pvs if "p" in s2 else vd, not on_dev)
        r_d = T.to_dev(r0)
        fn = getattr(L, f"QLA_{pc}_V_{var}{eq}_{s1}_times_{s2}")
        fn.restype = None
        args = [ctypes.c_void_p(r_d.data_ptr()), ctypes.c_void_p(a_addr), ctypes.c_void_p(b_addr)]
        gd = T.to_dev(gang)
        if var == "x":
            args.append(ctypes.c_void_p(gd.data_ptr()))
        fn(*args, ctypes.c_int(n), ctypes.c_int(nd))
        qla.check(fn.__name__)
        want = r0.copy() if var == "v" else np.concatenate([r0, np.zeros((ns - n, 6), dt)])[:n].copy()
        T.ora_multi(want, ms, vs, n, eq, adja=int(s1.endswith("a")), idx_a=ia if "p" in s1 else None,
                    idx_b=ib if "p" in s2 else None, gang=gang if var == "x" else None)
        assert T.bits_equal(T.to_host(r_d), want), (var, eq, s1, s2, nd)
        del keep_a, keep_b


@pytest.mark.parametrize("pc,dt", PCS)
def test_large_fields_refill_every_stage_bit_exact(qla, cuda, pc, dt):
    """2,097,152-site fields: every block of the pipelined kernel refills each
    shared-memory stage many times.  Three map families (axpy with the
    destination read, a gathered M*V, spin projection) must stay
    bit-identical to the oracle on two calls in a row."""
    rng = np.random.default_rng(91)
    n = 1 << 21
    ns_ = getattr(qla, pc)
    d = T.gaussian_field(rng, n, 12, dt)
    p = T.gaussian_field(rng, n, 12, dt)
    m = T.gaussian_field(rng, n, 9, dt)
    v = T.gaussian_field(rng, n, 3, dt)
    idx = _perm(rng, n)
    s = float(np.array(0.37, dtype=dt))
    d_d, p_d, m_d, v_d, i_d = T.to_dev(d), T.to_dev(p), T.to_dev(m), T.to_dev(v), T.to_dev(idx)
    for _ in range(2):
        x_d = T.to_dev(d)
        ns_.D_vpeq_r_times_D(x_d, s, p_d, n)
        want = d.copy()
        T.ora_rtimes(want, s, p, n, 12, "peq")
        assert T.bits_equal(T.to_host(x_d), want)
        r_d = T.to_dev(np.zeros((n, 6), dt))
        ns_.V_eq_M_times_xV(r_d, m_d, v_d, i_d, n)
        want = np.zeros((n, 6), dt)
        T.ora_lmult(want, m, v, n, 1, "eq", idx_b=idx)
        assert T.bits_equal(T.to_host(r_d), want)
        h_d = T.to_dev(np.zeros((n, 12), dt))
        ns_.H_veq_spproj_D(h_d, d_d, 2, -1, n)
        want = np.zeros((n, 12), dt)
        T.ora_spproj(want, d, n, 2, -1, "eq")
        assert T.bits_equal(T.to_host(h_d), want)
