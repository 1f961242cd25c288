"""GPU parity of the QLA_FN_ / QLA_DFN_ and QLA_DN_ entry points (colour
count nc at run time) against the oracle, through the C-ABI, for every
compiled nc (2, 3, 4, 8; matrix functions at nc = 2 by the templates'
two-colour closed forms).  Linear ops and the
matrix functions on the templates' generic paths (Pade exp, Newton sqrt,
Gauss-Jordan inverse, LU det, restated in float for FN and in double for DN)
must be bit-identical; reductions follow the tolerances of
tests/test_gpu_reductions.py."""
import itertools

import numpy as np
import pytest

import qla_testlib as T

pytestmark = pytest.mark.gpu

NCS = [2, 3, 4, 8]
# (library, site precision, reduction library returning double)
PRECS = [("FN", np.float32, "DFN"), ("DN", np.float64, "DN")]


def ncplx(t, nc):
    return {"V": nc, "H": 2 * nc, "D": 4 * nc, "M": nc * nc}[t]


def ncol(t, nc):
    return {"V": 1, "H": 2, "D": 4, "M": nc}[t]


@pytest.mark.parametrize("lib,dt,rlib", PRECS)
@pytest.mark.parametrize("nc", NCS)
def test_fn_lmult(qla, nc, lib, dt, rlib):
    rng = np.random.default_rng(50 + nc)
    ns_ = getattr(qla, lib)
    cb = 2 * np.dtype(dt).itemsize  # bytes per complex number
    n, ns = 1003, 1100
    idx = rng.integers(0, ns, n).astype(np.int32)
    gang = rng.permutation(n).astype(np.int32)
    a = rng.standard_normal((ns, 2 * nc * nc)).astype(dt)
    ad = T.to_dev(a)
    pa = T.ptr_array(ad, idx, cb * nc * nc)
    for dest in ("V", "H", "D", "M"):
        b = rng.standard_normal((ns, 2 * ncplx(dest, nc))).astype(dt)
        r0 = rng.standard_normal((n, 2 * ncplx(dest, nc))).astype(dt)
        bd = T.to_dev(b)
        pb = T.ptr_array(bd, idx[::-1].copy(), cb * ncplx(dest, nc))
        src2s = [(dest, 0), ("p" + dest, 0)] + ([("Ma", 1)] if dest == "M" else [])
        for var, eq, s1, (s2, adjb) in itertools.product(["v", "x"], T.EQOPS, ["M", "Ma", "pM"], src2s):
            if dest != "V" and var == "x" and eq not in ("eq", "meq"):
                continue
            r_d = T.to_dev(r0)
            args = [nc, r_d, pa if s1.startswith("p") else ad, pb if s2.startswith("p") else bd]
            if var == "x":
                args.append(T.to_dev(gang))
            getattr(ns_, f"{dest}_{var}{eq}_{s1}_times_{s2}")(*args, n)
            want = r0.copy()
            T.ora_lmult(want, a, b, n, ncol(dest, nc), eq, adja=int(s1.endswith("a")), adjb=adjb,
                        idx_a=idx if s1.startswith("p") else None,
                        idx_b=idx[::-1].copy() if s2.startswith("p") else None,
                        gang=gang if var == "x" else None, nc=nc)
            assert T.bits_equal(T.to_host(r_d), want), (lib, nc, dest, var, eq, s1, s2)
        r_d = T.to_dev(r0)
        ns_.__getattr__(f"{dest}_peq_M_times_x{dest}")(nc, r_d, ad, bd, T.to_dev(idx), n)
        want = r0.copy()
        T.ora_lmult(want, a, b, n, ncol(dest, nc), "peq", idx_b=idx, nc=nc)
        assert T.bits_equal(T.to_host(r_d), want), (nc, dest, "xb")


@pytest.mark.parametrize("lib,dt,rlib", PRECS)
@pytest.mark.parametrize("nc", NCS)
def test_fn_spin_rtimes_copy_reductions(qla, nc, lib, dt, rlib):
    rng = np.random.default_rng(60 + nc)
    ns_, rns = getattr(qla, lib), getattr(qla, rlib)
    n = 2049
    d = rng.standard_normal((n, 8 * nc)).astype(dt)
    h = rng.standard_normal((n, 4 * nc)).astype(dt)
    dd, hd = T.to_dev(d), T.to_dev(h)
    for eq, mu, sign in itertools.product(T.EQOPS, range(5), (1, -1)):
        r_d = T.to_dev(h)
        ns_.__getattr__(f"H_v{eq}_spproj_D")(nc, r_d, dd, mu, sign, n)
        want = h.copy()
        T.ora_spproj(want, d, n, mu, sign, eq, nc=nc)
        assert T.bits_equal(T.to_host(r_d), want), ("spproj", nc, eq, mu, sign)
        r_d = T.to_dev(d)
        ns_.__getattr__(f"D_v{eq}_sprecon_H")(nc, r_d, hd, mu, sign, n)
        want = d.copy()
        T.ora_sprecon(want, h, n, mu, sign, eq, nc=nc)
        assert T.bits_equal(T.to_host(r_d), want), ("sprecon", nc, eq, mu, sign)
    for t in ("V", "H", "D", "M"):
        x = rng.standard_normal((n, 2 * ncplx(t, nc))).astype(dt)
        y = rng.standard_normal((n, 2 * ncplx(t, nc))).astype(dt)
        xd, yd = T.to_dev(x), T.to_dev(y)
        for eq in T.EQOPS:
            r_d = T.to_dev(y)
            ns_.__getattr__(f"{t}_v{eq}_r_times_{t}")(nc, r_d, -0.375, xd, n)
            want = y.copy()
            T.ora_rtimes(want, -0.375, x, n, ncplx(t, nc), eq)
            assert T.bits_equal(T.to_host(r_d), want), ("rtimes", nc, t, eq)
        r_d = T.to_dev(y)
        ns_.__getattr__(f"{t}_vmeq_{t}")(nc, r_d, xd, n)
        assert T.bits_equal(T.to_host(r_d), y - x)
        exact = T.ora_norm2(x, n, ncplx(t, nc), exact=True)
        got = rns.__getattr__(f"r_veq_norm2_{t}")(nc, None, xd, n)
        assert abs(got - exact) <= 1e-12 * exact
        if lib == "FN":
            gotf = ns_.__getattr__(f"r_veq_norm2_{t}")(nc, None, xd, n)
            assert abs(gotf - exact) <= 6e-8 * exact
        ed = T.ora_dot(x, y, n, ncplx(t, nc), exact=True)
        gd = rns.__getattr__(f"c_veq_{t}_dot_{t}")(nc, None, xd, yd, n)
        assert abs(gd - ed) <= 1e-12 * max(1.0, abs(ed)) * 4


@pytest.mark.parametrize("lib,dt,rlib", PRECS)
@pytest.mark.parametrize("nc", [3, 4, 8])
def test_fn_matrix_functions_bit_exact(qla, nc, lib, dt, rlib):
    rng = np.random.default_rng(70 + nc)
    n = 4099 if nc < 8 else 1031
    gen = (rng.standard_normal((n, 2 * nc * nc)) * (0.4 if nc < 8 else 0.25)).astype(dt)
    pos = T.positive_hermitian_inputs(rng, n, dt, nc=nc)
    for fname, src in (("exp", gen), ("sqrt", pos), ("inverse", gen), ("det", gen)):
        nout = 1 if fname == "det" else nc * nc
        r_d = T.to_dev(np.zeros((n, 2 * nout), dt))
        dest = "C" if fname == "det" else "M"
        getattr(qla, lib).__getattr__(f"{dest}_veq_{fname}_M")(nc, r_d, T.to_dev(src), n)
        assert T.bits_equal(T.to_host(r_d), T.ora_mfunc(src, n, fname, nc=nc)), (lib, nc, fname)


@pytest.mark.parametrize("lib,dt,rlib", PRECS)
@pytest.mark.parametrize("nc", [3, 4, 8])
def test_fn_remaining_matrix_functions(qla, nc, lib, dt, rlib):
    """invsqrt, log, M^-1 V and M^-1 M take the templates' generic paths in
    float at every nc: bit-identical (log up to the host libm's log of
    |A|_F on the diagonal).  expA / expTA / sqrtPH / invsqrtPH take the exp and
    Newton paths at nc != 3 (bit-identical) and the FP64 closed forms at
    nc = 3 (FN: the F3 tolerance, the FP32 test rule against the FP64 value
    of the promoted input; DN: <= 1e-11 of max(1, |A|_F^2) against the
    oracle's double closed forms); eigenvalues take the closed forms at
    nc = 3 and the templates' Hessenberg + double-shift QR path
    (bit-identical) otherwise."""
    rng = np.random.default_rng(80 + nc)
    n = 2053 if nc < 8 else 521
    gen = (rng.standard_normal((n, 2 * nc * nc)) * (0.4 if nc < 8 else 0.25)).astype(dt)
    pos = T.positive_hermitian_inputs(rng, n, dt, nc=nc)
    z = T.to_complex(gen.astype(np.float64), nc)
    ah = T.from_complex(0.5 * (z - np.conj(np.transpose(z, (0, 2, 1)))), dt)
    herm = T.hermitian_inputs(rng, n, dt, nc=nc)
    cases = [("invsqrt", pos), ("log", pos), ("expA", ah), ("expTA", ah), ("sqrtPH", pos), ("invsqrtPH", pos),
             ("eigenvalsH", pos), ("eigenvalsH", herm), ("eigenvals", gen)]
    for fname, src in cases:
        nout = nc if fname.startswith("eigen") else nc * nc
        dest = "V" if fname.startswith("eigen") else "M"
        r_d = T.to_dev(np.zeros((n, 2 * nout), dt))
        getattr(qla, lib).__getattr__(f"{dest}_veq_{fname}_M")(nc, r_d, T.to_dev(src), n)
        got = T.to_host(r_d)
        closed = nc == 3 and fname not in ("invsqrt", "log")
        if closed and lib == "DN":
            want = T.ora_mfunc(src, n, fname, nc=nc)
            scale = np.maximum(1.0, np.sum(src.astype(np.float64) ** 2, axis=1))[:, None]
            assert np.all(np.abs(got - want) <= 1e-11 * scale), (lib, nc, fname)
        elif closed:
            want = T.ora_mfunc(src.astype(np.float64), n, fname, nc=nc)
            ok, nbad = T.qla_close(got, want, dt)
            assert ok, (nc, fname, nbad)
        elif fname == "log":
            want = T.ora_mfunc(src, n, fname, nc=nc)
            ok, nbad = T.qla_close(got, want, dt, nabs=2, nrel=2)
            assert ok, (nc, fname, nbad)
            assert np.mean(np.all(got == want, axis=1)) > 0.99
        else:
            assert T.bits_equal(got, T.ora_mfunc(src, n, fname, nc=nc)), (nc, fname)
    for t, nb in (("V", 1), ("M", nc)):
        b = rng.standard_normal((n, 2 * nc * nb)).astype(dt)
        ib = rng.permutation(n).astype(np.int32)
        r_d = T.to_dev(np.zeros((n, 2 * nc * nb), dt))
        b_d = T.to_dev(b)
        pb = T.ptr_array(b_d, ib, 2 * np.dtype(dt).itemsize * nc * nb)
        getattr(qla, lib).__getattr__(f"{t}_veq_M_inverse_p{t}")(nc, r_d, T.to_dev(gen), pb, n)
        assert T.bits_equal(T.to_host(r_d), T.ora_minv(gen, b, n, nb, nc=nc, idx_b=ib)), (nc, t)


@pytest.mark.parametrize("lib,dt,rlib", PRECS)
def test_fn_two_colour_matrix_functions(qla, lib, dt, rlib):
    """nc = 2 takes the templates' two-colour closed forms (the oracle's are
    pinned to the reference's F2 / D2 and FN / DN builds).  sqrt, invsqrt,
    sqrtPH, invsqrtPH, inverse, det, eigenvalues and a^-1 b are bit-identical,
    zero and singular inputs included; exp, log, expA and expTA call CUDA's
    sinh / exp / sincos / log / atan2 where the reference calls the host
    libm: within 64 eps of max(1, max |r|) per site (the test prints the
    fraction of sites that are bit-identical)."""
    rng = np.random.default_rng(92)
    n, nc = 4099, 2
    gen = (rng.standard_normal((n, 8)) * 0.7).astype(dt)
    z = T.to_complex(gen.astype(np.float64), nc)
    ah = T.from_complex(0.5 * (z - np.conj(np.transpose(z, (0, 2, 1)))), dt)
    aht = T.from_complex(T.to_complex(ah.astype(np.float64), nc)
                         + 1j * rng.uniform(-1, 1, n)[:, None, None] * np.eye(2), dt)
    pos = T.positive_hermitian_inputs(rng, n, dt, nc=nc)
    herm = T.hermitian_inputs(rng, n, dt, nc=nc)
    u = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
    rank1 = np.einsum("ni,nj->nij", u, np.conj(u))
    rank1[::7] = 0
    psd1 = T.from_complex(rank1, dt)
    scal = T.from_complex((rng.uniform(0.5, 2, n) + 1j * rng.uniform(-1, 1, n))[:, None, None] * np.eye(2), dt)
    exact = [("sqrt", pos), ("sqrt", gen), ("sqrt", psd1), ("invsqrt", pos), ("invsqrt", gen), ("inverse", gen),
             ("det", gen), ("det", psd1), ("sqrtPH", pos), ("sqrtPH", psd1), ("invsqrtPH", pos),
             ("eigenvals", gen), ("eigenvals", psd1), ("eigenvalsH", herm), ("eigenvalsH", psd1)]
    approx = [("exp", gen), ("exp", ah), ("exp", scal), ("log", pos), ("log", gen), ("log", scal),
              ("expA", aht), ("expA", ah), ("expTA", ah)]
    eps = np.finfo(dt).eps
    for k, (fname, src) in enumerate(exact + approx):
        dest = "C" if fname == "det" else "V" if fname.startswith("eigen") else "M"
        nout = {"C": 1, "V": 2, "M": 4}[dest]
        r_d = T.to_dev(np.zeros((n, 2 * nout), dt))
        getattr(qla, lib).__getattr__(f"{dest}_veq_{fname}_M")(nc, r_d, T.to_dev(src), n)
        got = T.to_host(r_d)
        want = T.ora_mfunc(src, n, fname, nc=nc)
        if k < len(exact):
            assert T.bits_equal(got, want), (lib, fname)
        else:
            scale = np.maximum(1.0, np.max(np.abs(want.astype(np.float64)), axis=1))[:, None]
            assert np.all(np.abs(got.astype(np.float64) - want) <= 64 * eps * scale), (lib, fname)
            print(f"{lib} nc=2 {fname}: sites bit-identical {np.mean(np.all(got == want, axis=1)):.4f}")
    for t, nb in (("V", 1), ("M", 2)):
        b = rng.standard_normal((n, 4 * nb)).astype(dt)
        ib = rng.permutation(n).astype(np.int32)
        r_d = T.to_dev(np.zeros((n, 4 * nb), dt))
        b_d = T.to_dev(b)
        pb = T.ptr_array(b_d, ib, 2 * np.dtype(dt).itemsize * nc * nb)
        getattr(qla, lib).__getattr__(f"{t}_veq_M_inverse_p{t}")(nc, r_d, T.to_dev(gen), pb, n)
        assert T.bits_equal(T.to_host(r_d), T.ora_minv(gen, b, n, nb, nc=nc, idx_b=ib)), (lib, t)


def test_fn_unsupported_nc_reports_error(qla):
    qla.clear_error()
    qla.lib().QLA_FN_V_veq_M_times_V(5, None, None, None, 10)
    code, msg = qla.last_error()
    assert code == 4 and "nc not compiled" in msg
    qla.clear_error()


@pytest.mark.parametrize("lib,dt,rlib", PRECS)
@pytest.mark.parametrize("nc", [2, 4])
def test_fn_fused_hop_terms(qla, nc, lib, dt, rlib):
    """{H,D}_*_spproj_{M,Ma,pM,pMa}_times_{D,pD}, D_*_sprecon_*_times_{H,pH},
    D_*_spproj_D and the int32-index forms at nc colours, against the oracle
    composition in the reference's order, bit for bit."""
    rng = np.random.default_rng(90 + nc)
    ns_ = getattr(qla, lib)
    cb = 2 * np.dtype(dt).itemsize
    n, ns = 301, 320
    a = rng.standard_normal((ns, 2 * nc * nc)).astype(dt)
    d_src = rng.standard_normal((ns, 8 * nc)).astype(dt)
    h_src = rng.standard_normal((ns, 4 * nc)).astype(dt)
    r0 = {"H": rng.standard_normal((ns, 4 * nc)).astype(dt), "D": rng.standard_normal((ns, 8 * nc)).astype(dt)}
    idx = rng.integers(0, ns, ns).astype(np.int32)
    gang = rng.permutation(n).astype(np.int32)
    ad, dd, hd = T.to_dev(a), T.to_dev(d_src), T.to_dev(h_src)
    pa = T.ptr_array(ad, idx, cb * nc * nc)
    pdd = T.ptr_array(dd, idx, cb * 4 * nc)
    phd = T.ptr_array(hd, idx, cb * 2 * nc)
    for (dest, kind), eq, s1, pb, var in itertools.product(
            [("H", "spproj"), ("D", "spproj"), ("D", "sprecon")], T.EQOPS, ["M", "Ma", "pMa"], [0, 1], ["v", "x"]):
        src = "D" if kind == "spproj" else "H"
        bsrc, bdev, bptr = (d_src, dd, pdd) if src == "D" else (h_src, hd, phd)
        mu, sign = (eq.count("e") + len(s1) + pb) % 5, (1 if var == "v" else -1)
        r_d = T.to_dev(r0[dest][:n])
        args = [nc, r_d, pa if s1.startswith("p") else ad, bptr if pb else bdev, mu, sign]
        if var == "x":
            args.append(T.to_dev(gang))
        getattr(ns_, f"{dest}_{var}{eq}_{kind}_{s1}_times_{'p' if pb else ''}{src}")(*args, n)
        want = r0[dest][:n].copy()
        aa = a[idx[:n]] if s1.startswith("p") else a[:n]
        T.ora_hop(want, np.ascontiguousarray(aa), bsrc, n, mu, sign, eq, dest, kind, adja=int(s1.endswith("a")),
                  idx_b=idx if pb else None, gang=gang if var == "x" else None, nc=nc)
        assert T.bits_equal(T.to_host(r_d), want), (lib, nc, dest, kind, var, eq, s1, pb, mu, sign)
    for (dest, kind), eq in itertools.product([("H", "spproj"), ("D", "spproj"), ("D", "sprecon")], T.EQOPS):
        src = "D" if kind == "spproj" else "H"
        bsrc, bdev = (d_src, dd) if src == "D" else (h_src, hd)
        r_d = T.to_dev(r0[dest][:n])
        ns_.__getattr__(f"{dest}_{eq}_{kind}_M_times_x{src}")(nc, r_d, ad, bdev, T.to_dev(idx), 2, -1, n)
        want = r0[dest][:n].copy()
        T.ora_hop(want, np.ascontiguousarray(a[:n]), bsrc, n, 2, -1, eq, dest, kind, idx_b=idx, nc=nc)
        assert T.bits_equal(T.to_host(r_d), want), (lib, nc, dest, kind, eq, "xb")
    for eq, mu in itertools.product(T.EQOPS, range(5)):
        r_d = T.to_dev(r0["D"][:n])
        ns_.__getattr__(f"D_v{eq}_spproj_D")(nc, r_d, dd, mu, 1, n)
        want = r0["D"][:n].copy()
        T.ora_hop(want, None, d_src, n, mu, 1, eq, "D", "spproj", nc=nc)
        assert T.bits_equal(T.to_host(r_d), want), (lib, nc, "Dspproj", eq, mu)


@pytest.mark.parametrize("lib,dt,rlib", PRECS)
@pytest.mark.parametrize("nc", [2, 4])
def test_fn_propagator_entry_points(qla, nc, lib, dt, rlib):
    """Every N-colour DiracPropagator product (M P, P M, P P with adjoint /
    pointer / gang / eqop forms) and spin trace at nc colours, bit-exact."""
    rng = np.random.default_rng(95 + nc)
    n, ns = 67, 71
    names = [e["name"] for e in qla.manifest() if e["pc"] == lib and e["family"] == "prop"]
    assert len(names) == 388
    data, cases = T.prop_cases(lib, names, nc, dt, rng, n, ns)
    cb = 2 * np.dtype(dt).itemsize
    dev = {k: T.to_dev(data[k]) for k in ("M", "P1", "P2")}
    rec = {"M": cb * nc * nc, "P1": cb * 16 * nc * nc, "P2": cb * 16 * nc * nc}
    ptrs_a = {k: T.ptr_array(v, data["ia"], rec[k]) for k, v in dev.items()}
    ptrs_b = {k: T.ptr_array(v, data["ib"], rec[k]) for k, v in dev.items()}
    gd = T.to_dev(data["gang"])
    L = qla.lib()
    bad = []
    for name, spec, want in cases:
        r_d = T.to_dev(spec["r0"])
        ka, pa = spec["a"]
        args = [nc, T.ptr_dev(r_d), T.ptr_dev(ptrs_a[ka] if pa else dev[ka])]
        if spec["b"] is not None:
            kb, pb = spec["b"]
            args.append(T.ptr_dev(ptrs_b[kb] if pb else dev[kb]))
        if spec["var"] == "x":
            args.append(T.ptr_dev(gd))
        getattr(L, name)(*args, n)
        if not T.bits_equal(T.to_host(r_d), want):
            bad.append(name)
    qla.check(f"{lib} prop nc={nc}")
    assert not bad, f"{len(bad)} mismatches, e.g. {bad[:6]}"


@pytest.mark.parametrize("lib,dt,rlib", PRECS)
@pytest.mark.parametrize("nc,nd", [(2, 3), (4, 11)])
def test_fn_multi_direction_sum(qla, nc, nd, lib, dt, rlib):
    """V_{v,x}{eqop}_n{p}M{a}_times_n{p}V at nc colours: the reference's
    per-direction rounding, nd = 11 in two launches, operand tables on the
    host and on the device, bit for bit."""
    import ctypes
    rng = np.random.default_rng(97 + nc)
    cb = 2 * np.dtype(dt).itemsize
    n, ns = 203, 220
    ms = [rng.standard_normal((ns, 2 * nc * nc)).astype(dt) for _ in range(nd)]
    vs = [rng.standard_normal((ns, 2 * nc)).astype(dt) for _ in range(nd)]
    r0 = rng.standard_normal((n, 2 * nc)).astype(dt)
    ia = rng.integers(0, ns, ns).astype(np.int32)
    ib = rng.integers(0, ns, ns).astype(np.int32)
    gang = rng.permutation(n).astype(np.int32)
    md = [T.to_dev(m) for m in ms]
    vd = [T.to_dev(v) for v in vs]
    pms = [T.ptr_array(m, ia, cb * nc * nc) for m in md]
    pvs = [T.ptr_array(v, ib, cb * nc) for v in vd]
    L = qla.lib()

    def table(ts, on_dev):
        addrs = np.array([t.data_ptr() for t in ts], dtype=np.int64)
        if on_dev:
            d = T.to_dev(addrs)
            return d, d.data_ptr()
        return addrs, addrs.ctypes.data

    gd = T.to_dev(gang)
    for var, eq, s1, s2 in itertools.product(["v", "x"], T.EQOPS, ["nM", "nMa", "npMa"], ["nV", "npV"]):
        on_dev = (eq in ("peq", "eqm"))
        keep_a, a_addr = table(pms if "p" in s1 else md, on_dev)
        keep_b, b_addr = table(pvs if "p" in s2 else vd, not on_dev)
        r_d = T.to_dev(r0)
        fn = getattr(L, f"QLA_{lib}_V_{var}{eq}_{s1}_times_{s2}")
        fn.restype = None
        args = [ctypes.c_int(nc), ctypes.c_void_p(r_d.data_ptr()), ctypes.c_void_p(a_addr), ctypes.c_void_p(b_addr)]
        if var == "x":
            args.append(ctypes.c_void_p(gd.data_ptr()))
        fn(*args, ctypes.c_int(n), ctypes.c_int(nd))
        qla.check(fn.__name__)
        want = r0.copy()
        T.ora_multi(want, ms, vs, n, eq, adja=int(s1.endswith("a")), idx_a=ia if "p" in s1 else None,
                    idx_b=ib if "p" in s2 else None, gang=gang if var == "x" else None, nc=nc)
        assert T.bits_equal(T.to_host(r_d), want), (lib, nc, var, eq, s1, s2, nd)
        del keep_a, keep_b
