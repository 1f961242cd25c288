"""GPU parity of the DiracPropagator products (M*P, P*M, P*P with every
adjoint / pointer / gang / eqop form) and the spin trace, bit-exact against
the oracle, through the C-ABI (every generated P entry point is called)."""
import re

import numpy as np
import pytest

import qla_testlib as T

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64)])
def test_all_propagator_entry_points(qla, pc, dt):
    rng = np.random.default_rng(123)
    n, ns = 193, 211
    m = T.haar_su3(rng, ns, dt)
    p1 = T.gaussian_field(rng, ns, 144, dt)
    p2 = T.gaussian_field(rng, ns, 144, dt)
    r0p = T.gaussian_field(rng, ns, 144, dt)
    r0m = T.gaussian_field(rng, ns, 9, dt)
    ia = rng.integers(0, ns, ns).astype(np.int32)
    ib = rng.integers(0, ns, ns).astype(np.int32)
    gang = rng.permutation(n).astype(np.int32)
    e = 8 if dt == np.float32 else 16
    dev = {"M": T.to_dev(m), "P1": T.to_dev(p1), "P2": T.to_dev(p2)}
    ptrs_a = {k: T.ptr_array(v, ia, e * (9 if k == "M" else 144)) for k, v in dev.items()}
    ptrs_b = {k: T.ptr_array(v, ib, e * (9 if k == "M" else 144)) for k, v in dev.items()}
    names = [x["name"] for x in qla.manifest() if x["family"] == "prop" and x["name"].startswith(f"QLA_{pc}_")]
    assert len(names) == 388  # 48 products x 4 eqops x (v, x) + spintrace (P, pP) x (v, x)
    gd = T.to_dev(gang)
    for name in names:
        short = name[len(f"QLA_{pc}_"):]
        mt = re.match(r"M_([vx])eq_spintrace_(p?)P$", short)
        if mt:
            var, pa = mt.groups()
            r_d = T.to_dev(r0m[:n])
            args = [r_d, ptrs_a["P1"] if pa else dev["P1"]] + ([gd] if var == "x" else []) + [n]
            getattr(getattr(qla, pc), short)(*args)
            want = r0m[:n].copy()
            T.ora_prop("TRACE", want, p1, None, n, "eq", idx_a=ia if pa else None, gang=gang if var == "x" else None)
            assert T.bits_equal(T.to_host(r_d), want), name
            continue
        var, eq, pa, ta, ca, pb, tb, cb = re.match(
            r"P_([vx])(eq|peq|meq|eqm)_(p?)(M|P)(a?)_times_(p?)(M|P)(a?)$", short).groups()
        ka = "M" if ta == "M" else "P1"
        kb = "M" if tb == "M" else "P2"
        r_d = T.to_dev(r0p[:n])
        args = [r_d, ptrs_a[ka] if pa else dev[ka], ptrs_b[kb] if pb else dev[kb]]
        if var == "x":
            args.append(gd)
        getattr(getattr(qla, pc), short)(*args, n)
        want = r0p[:n].copy()
        T.ora_prop(ta + tb, want, m if ta == "M" else p1, m if tb == "M" else p2, n, eq, ca=int(bool(ca)),
                   cb=int(bool(cb)), idx_a=ia if pa else None, idx_b=ib if pb else None,
                   gang=gang if var == "x" else None)
        assert T.bits_equal(T.to_host(r_d), want), name


@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64)])
@pytest.mark.parametrize("n", [1, 7, 20011])
def test_propagator_products_many_tiles_and_tiny_fields(qla, pc, dt, n):
    """The contiguous P*P, M*P and P*M kernels (bulk-copy pipeline) at sizes
    where persistent blocks walk many tiles (stage ring refilled many times;
    20,011 sites ends in a partial tile, which M*P and P*M hand to the direct
    kernel) and at fewer sites than one tile, every eqop and adjoint."""
    rng = np.random.default_rng(124 + n)
    p1 = T.gaussian_field(rng, n, 144, dt)
    p2 = T.gaussian_field(rng, n, 144, dt)
    m = T.gaussian_field(rng, n, 9, dt)
    r0 = T.gaussian_field(rng, n, 144, dt)
    d1, d2, dm = T.to_dev(p1), T.to_dev(p2), T.to_dev(m)
    for ta, tb in (("P", "P"), ("M", "P"), ("P", "M")):
        for eq in ("eq", "peq", "meq", "eqm"):
            for ca in ("", "a"):
                for cb in ("", "a"):
                    name = f"P_v{eq}_{ta}{ca}_times_{tb}{cb}"
                    xa, xb = (m if ta == "M" else p1), (m if tb == "M" else p2)
                    da, db = (dm if ta == "M" else d1), (dm if tb == "M" else d2)
                    r_d = T.to_dev(r0)
                    getattr(getattr(qla, pc), name)(r_d, da, db, n)
                    want = r0.copy()
                    T.ora_prop(ta + tb, want, xa, xb, n, eq, ca=int(bool(ca)), cb=int(bool(cb)))
                    assert T.bits_equal(T.to_host(r_d), want), (name, n)
    assert qla.device_error() == 0
