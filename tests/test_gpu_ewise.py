"""GPU parity of the element-wise families, the site-local dot products and
norms, and the ColorVector outer product: every generated entry point (F3 and
D3, all eqops, pointer and gang forms) through the C-ABI against the oracle,
bit for bit.  The oracle is pinned to the reference library entry point by
entry point (tests/test_oracle_pin.py)."""
import json
import os

import numpy as np
import pytest

import qla_testlib as T

pytestmark = pytest.mark.gpu

MANIFEST = os.path.join(T.REPO, "qla_b200", "gen", "api_manifest.json")


def _entries(pc):
    man = json.load(open(MANIFEST))
    return [e for e in man if e["pc"] == pc and (e["family"].startswith("ewise") or e["family"] == "ldot")]


def _rec_bytes(letter, dt):
    return np.dtype(dt).itemsize * (1 if letter == "R" else 2 if letter == "C" else 2 * T.NE3[letter])


@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64)])
def test_every_elementwise_entry_point(qla, pc, dt):
    rng = np.random.default_rng(202)
    L = qla.lib()
    n, ns = 61, 67
    bad, count = [], 0
    for j, e in enumerate(_entries(pc)):
        ins, idx, gang = T.ewise_inputs(e, rng, dt, n, ns)
        want = T.ewise_oracle(e, ins, idx, gang, n)
        keep, args = [], []
        r_d = None
        plan, kw = T.ewise_oracle_plan(e)
        const_a = plan == "ewise" and kw["scal_kind"] == 1
        for t, name in zip(e["ctypes"], e["params"]):
            if name == "n":
                args.append(len(gang) if gang is not None else n)
            elif name == "index":
                g = T.to_dev(gang)
                keep.append(g)
                args.append(T.ptr_dev(g))
            elif name == "r":
                r_d = T.to_dev(ins["r"][2])
                args.append(T.ptr_dev(r_d))
            else:
                letter, is_ptr, arr = ins[name]
                if is_ptr:
                    base = T.to_dev(arr)
                    pa = T.ptr_array(base, idx[name], _rec_bytes(letter, dt))
                    keep += [base, pa]
                    args.append(T.ptr_dev(pa))
                elif name == "a" and const_a:
                    # a constant: host memory on even entries, device memory on odd ones
                    if j % 2 == 0:
                        keep.append(arr)
                        args.append(T.ptr(arr))
                    else:
                        d = T.to_dev(arr)
                        keep.append(d)
                        args.append(T.ptr_dev(d))
                else:
                    d = T.to_dev(arr)
                    keep.append(d)
                    args.append(T.ptr_dev(d))
        getattr(L, e["name"])(*args)
        count += 1
        got = T.to_host(r_d)
        if not T.bits_equal(got, want):
            bad.append(e["name"])
    qla.check("elementwise")
    assert count > 1800
    assert not bad, f"{len(bad)} mismatches, e.g. {bad[:8]}"


@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64)])
def test_elementwise_large_fields(qla, pc, dt):
    """A few representative forms on 2^20-site fields (many grid-stride
    iterations per thread)."""
    rng = np.random.default_rng(203)
    L = qla.lib()
    n = 1 << 20
    names = [f"QLA_{pc}_D_vpeq_c_times_D", f"QLA_{pc}_M_veq_Ca_times_Ma", f"QLA_{pc}_V_veq_c_times_V_plus_V",
             f"QLA_{pc}_C_vpeq_D_dot_D", f"QLA_{pc}_R_veq_norm2_M", f"QLA_{pc}_M_vmeq_V_times_Va"]
    man = {e["name"]: e for e in json.load(open(MANIFEST))}
    for nm in names:
        e = man[nm]
        ins, idx, gang = T.ewise_inputs(e, rng, dt, n, n)
        want = T.ewise_oracle(e, ins, idx, gang, n)
        keep, args = [], []
        for t, name in zip(e["ctypes"], e["params"]):
            if name == "n":
                args.append(n)
            elif name == "r":
                r_d = T.to_dev(ins["r"][2])
                args.append(T.ptr_dev(r_d))
            else:
                d = T.to_dev(ins[name][2])
                keep.append(d)
                args.append(T.ptr_dev(d))
        getattr(L, nm)(*args)
        assert T.bits_equal(T.to_host(r_d), want), nm
    qla.check("elementwise large")


@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64)])
def test_site_local_reductions_tiles_and_alignment(qla, pc, dt):
    """The staged path of the site-local dot products and norms (tiles of
    records copied into shared memory) on lengths that leave a partial last
    tile, and the same calls on operands that start half a complex number
    past an aligned address: bit-identical to the oracle either way."""
    import ctypes
    rng = np.random.default_rng(204)
    L = qla.lib()
    man = {e["name"]: e for e in json.load(open(MANIFEST))}
    names = [f"QLA_{pc}_C_vpeq_D_dot_D", f"QLA_{pc}_R_veq_norm2_P", f"QLA_{pc}_C_veq_P_dot_P",
             f"QLA_{pc}_C_veq_M_dot_M", f"QLA_{pc}_R_veq_re_P_dot_P"]
    item = np.dtype(dt).itemsize
    for nm in names:
        e = man[nm]
        for n in (1, 33, 1031):
            ins, idx, gang = T.ewise_inputs(e, rng, dt, n, n)
            want = T.ewise_oracle(e, ins, idx, gang, n)
            for shift in (0, 1):
                keep, args = [], []
                for t, name in zip(e["ctypes"], e["params"]):
                    if name == "n":
                        args.append(n)
                    elif name == "r":
                        r_d = T.to_dev(ins["r"][2])
                        args.append(T.ptr_dev(r_d))
                    else:
                        flat = np.concatenate([np.zeros(shift, dt), ins[name][2].ravel()])
                        d = T.to_dev(flat)
                        keep.append(d)
                        args.append(ctypes.c_void_p(d.data_ptr() + shift * item))
                getattr(L, nm)(*args)
                assert T.bits_equal(T.to_host(r_d), want), (nm, n, shift)
    qla.check("site-local reductions")
