"""GPU parity of the site-field families through the C-ABI: constant,
diagonal and zero fills, copymask, component / colour-column / Dirac-vector
extraction and insertion, gamma multiplication (every mu), traces and the
antihermitian part bit for bit against the oracle; the global reductions of
DiracPropagators and adjoint-form products and the global sums against the
oracle's reference-order sums within the stated tolerance.  The oracle is
pinned to the reference library entry point by entry point
(tests/test_oracle_pin.py).

Tolerance of the global reductions and sums: the GPU forms each site's sum in
double in the reference's element order and adds the sites in double-double;
the reference adds every term into one double.  Both are rounded to the site
precision at the end.  Against the reference-order value v over terms t:
  |gpu - v| <= 2 ulp(v) of the output precision + 1e-13 * sum |t|  (F3)
  |gpu - v| <= 1e-13 * sum |t|                                      (D3)
"""
import json
import os

import numpy as np
import pytest

import qla_testlib as T

pytestmark = pytest.mark.gpu

MANIFEST = os.path.join(T.REPO, "qla_b200", "gen", "api_manifest.json")


def _man():
    return json.load(open(MANIFEST))


def _dev_args(e, ins, idx, gang, n, dt, ints, keep, host_const=False):
    """C-ABI arguments with every field in device memory; returns (args, r_dev)."""
    args, r_d = [], None
    for t, name in zip(e["ctypes"], e["params"]):
        if name == "n":
            args.append(len(gang) if gang is not None else n)
        elif name == "index":
            g = T.to_dev(gang)
            keep.append(g)
            args.append(T.ptr_dev(g))
        elif t == "int":
            args.append(ints[name])
        elif name == "r":
            r_d = T.to_dev(ins["r"][2])
            args.append(T.ptr_dev(r_d))
        else:
            letter, is_ptr, arr = ins[name]
            if is_ptr:
                base = T.to_dev(arr)
                pa = T.ptr_array(base, idx[name], T.rec_bytes(letter, dt))
                keep += [base, pa]
                args.append(T.ptr_dev(pa))
            elif host_const:
                keep.append(arr)
                args.append(T.ptr(arr))
            else:
                d = T.to_dev(arr)
                keep.append(d)
                args.append(T.ptr_dev(d))
    return args, r_d


@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64)])
def test_every_sitefield_entry_point(qla, pc, dt):
    rng = np.random.default_rng(301)
    L = qla.lib()
    n, ns = 61, 67
    bad, count = [], 0
    for j, e in enumerate(x for x in _man() if x["pc"] == pc and x["family"] in T.SF_FAMILIES):
        reps = 16 if e["family"] == "gamma" else 1
        for rep in range(reps):
            ins, idx, gang, ints = T.sitefield_inputs(e, rng, dt, n, ns)
            if "mu" in ints:
                ints["mu"] = rep
            want = T.sitefield_oracle(e, ins, idx, gang, n, ints)
            keep = []
            # fill constants: host memory on even entries, device memory on odd ones
            host_const = e.get("op") in ("fill", "diagfill") and j % 2 == 0
            args, r_d = _dev_args(e, ins, idx, gang, n, dt, ints, keep, host_const)
            getattr(L, e["name"])(*args)
            count += 1
            if not T.bits_equal(T.to_host(r_d), want):
                bad.append((e["name"], ints))
    qla.check("sitefield")
    assert count > 300
    assert not bad, f"{len(bad)} mismatches, e.g. {bad[:8]}"


def test_gamma_index_outside_range_leaves_r_and_records_error(qla):
    L = qla.lib()
    rng = np.random.default_rng(302)
    a = T.to_dev(rng.standard_normal((8, 24)).astype(np.float32))
    r0 = rng.standard_normal((8, 24)).astype(np.float32)
    r = T.to_dev(r0)
    qla.clear_error()
    L.QLA_F3_D_veq_gamma_times_D(T.ptr_dev(r), T.ptr_dev(a), 16, 8)
    assert qla.last_error()[0] == 4  # QLAGPU_ERR_ARG
    qla.clear_error()
    assert T.bits_equal(T.to_host(r), r0)


def test_component_index_outside_range_is_refused(qla):
    L = qla.lib()
    rng = np.random.default_rng(303)
    a = T.to_dev(rng.standard_normal((8, 12)).astype(np.float32))
    r0 = np.zeros((8, 2), np.float32)
    r = T.to_dev(r0)
    qla.clear_error()
    # a HalfFermion has spins 0 and 1 only
    L.QLA_F3_C_veq_elem_H(T.ptr_dev(r), T.ptr_dev(a), 1, 2, 8)
    assert qla.last_error()[0] == 4
    qla.clear_error()
    assert T.bits_equal(T.to_host(r), r0)


def _terms_abs(e, ins, idx, gang, n):
    """sum of |terms| of a global reduction / sum (the error scale)."""
    a = ins["a"][2].astype(np.float64)
    k = np.asarray(gang if gang is not None else np.arange(n), np.int64)
    ka = idx["a"][k] if "a" in idx else k
    if e["family"] == "gsum":
        return np.abs(a[ka]).sum(axis=0)
    b = ins["b"][2].astype(np.float64) if "b" in ins else a
    kb = (idx["b"][k] if "b" in idx else k) if "b" in ins else ka
    # sum_e |a_pi(e)| |b_e| <= (sum |a|^2 + sum |b|^2) / 2 for any pairing pi
    return np.full(2, 0.5 * (np.square(a[ka]).sum() + np.square(b[kb]).sum()))


@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64), ("DF3", np.float32)])
@pytest.mark.parametrize("n", [1, 61, 4099])
def test_global_p_reductions_and_sums(qla, cuda, pc, dt, n):
    rng = np.random.default_rng(304 + n)
    L = qla.lib()
    ns = n + 7
    bad, count = [], 0
    for e in (x for x in _man() if x["pc"] == pc and x["family"] in ("gred", "gsum")):
        ins, idx, gang, _ = T.sitefield_inputs(e, rng, dt, n, ns)
        if e["family"] == "gred":
            out = T.gred_oracle(e, ins, idx, gang, n)
            want = out[:1] if e["dest"] == "r" else out
        else:
            want = T.gsum_oracle(e, ins, idx, gang, n).astype(np.float64)
        scale = _terms_abs(e, ins, idx, gang, n)[: len(want)]
        odt = np.float64 if e.get("out") == "double" else dt
        eps = np.finfo(dt).eps
        tol = 1e-13 * scale + (4 * eps * np.abs(want) if odt == np.float32 else 0)
        if dt == np.float32 and e.get("kind") == "LD_NORM2":
            # the reference rounds each |a_e|^2 to float before adding it
            tol = tol + 2 * eps * scale
        for dev_out in (False, True):
            keep = []
            args, _ = _dev_args(e, ins, idx, gang, n, dt, {}, keep)
            if dev_out:
                r_d = cuda.zeros(len(want), dtype=cuda.float32 if odt == np.float32 else cuda.float64, device="cuda")
                args[0] = T.ptr_dev(r_d)
                getattr(L, e["name"])(*args)
                got = r_d.cpu().numpy().astype(np.float64)
            else:
                r_h = np.zeros(len(want), odt)
                args[0] = T.ptr(r_h)
                getattr(L, e["name"])(*args)
                got = r_h.astype(np.float64)
            count += 1
            if np.any(np.abs(got - want) > tol):
                bad.append((e["name"], dev_out, float(np.max(np.abs(got - want) / np.maximum(scale, 1e-300)))))
    qla.check("global P reductions / sums")
    assert count == 112
    assert not bad, f"{len(bad)} outside tolerance, e.g. {bad[:6]}"


def test_global_sums_are_deterministic_on_large_fields(qla, cuda):
    """2^18 DiracPropagator sites (300 MB F3): the sum is the same bit pattern
    on repeated calls (fixed block-order fold), and within tolerance of an
    exact float64 fsum of the components."""
    import math
    rng = np.random.default_rng(305)
    L = qla.lib()
    n = 1 << 18
    a = rng.standard_normal((n, 288)).astype(np.float32)
    ad = T.to_dev(a)
    outs = []
    for _ in range(3):
        r = np.zeros(288, np.float32)
        L.QLA_F3_p_veq_sum_P(T.ptr(r), T.ptr_dev(ad), n)
        outs.append(r)
    assert all(T.bits_equal(outs[0], o) for o in outs[1:])
    exact = np.array([math.fsum(a[:, c].astype(np.float64)) for c in range(0, 288, 37)])
    got = outs[0][::37].astype(np.float64)
    scale = np.abs(a[:, ::37]).astype(np.float64).sum(axis=0)
    assert np.all(np.abs(got - exact) <= 4 * np.finfo(np.float32).eps * np.abs(exact) + 1e-13 * scale)
    qla.check("large sum")


def test_precision_conversions(qla):
    """QLA_DF3_X_*eq_X and QLA_FD3_X_*eq_X, every entry point, bit for bit."""
    rng = np.random.default_rng(306)
    L = qla.lib()
    n, ns = 61, 67
    bad = []
    entries = [x for x in _man() if x["family"] == "convert" and x["pc"] == "DF3"]
    for e in entries:
        ins, idx, gang = T.convert_inputs(e, rng, n, ns)
        want = T.convert_oracle(e, ins, idx, gang, n)
        src_dt = ins["a"][2].dtype
        keep = []
        args, r_d = _dev_args(e, ins, idx, gang, n, src_dt, {}, keep)
        getattr(L, e["name"])(*args)
        if not T.bits_equal(T.to_host(r_d), want):
            bad.append(e["name"])
    qla.check("conversions")
    assert len(entries) == 40
    assert not bad, bad[:8]
