"""GPU parity of the real / complex / integer field libraries (QLA_F_,
QLA_D_, QLA_DF_ / QLA_FD_) through the C-ABI, every entry point against the
oracle (pinned to the reference library,
tests/test_oracle_pin.py::test_oracle_real_complex_field_libraries_match_reference_library).

Tolerances, per kind of operation:
  * arithmetic, conversions, comparisons, rounding, masks, sqrt / fabs /
    ceil / floor, fmod, ldexp, complex division and square root, site-local
    dot products: bit-identical;
  * the transcendental functions (sin ... tanh, exp, log, log10, pow, atan2,
    arg, cexp, cexpi, clog): CUDA's implementations against the host libm,
    within 4 units in the last place of the result (the test prints the
    fraction that is bit-identical);
  * global reductions and sums: the GPU adds the sites in double-double, the
    reference in one double: |gpu - ref| <= 1e-13 * sum|terms| plus 4 ulp of
    a float result; the F and DF libraries' complex norm2 also carries the
    reference's float rounding of each |a|^2 (2 float eps * sum|terms|).
"""
import numpy as np
import pytest

import qla_testlib as T

pytestmark = pytest.mark.gpu


def _dev_args(e, ins, idx, gang, n, keep, host_const):
    args, r_d = [], None
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
                pa = T.ptr_array(base, idx[name], arr.itemsize * (2 if letter == "C" else 1))
                keep += [base, pa]
                args.append(T.ptr_dev(pa))
            elif host_const and e.get("opnds") and [name, letter.lower()] in e["opnds"]:
                keep.append(arr)
                args.append(T.ptr(arr))
            else:
                d = T.to_dev(arr)
                keep.append(d)
                args.append(T.ptr_dev(d))
    return args, r_d


def _scale(e, ins):
    a = np.abs(ins["a"][2].astype(np.float64))
    if e.get("plan") == "gsum" or e.get("spec") == "SR_SUM":
        return a.sum()
    if "b" in ins and e.get("spec") not in ("LD_NORM2", "SR_NORM2"):
        b = np.abs(ins["b"][2].astype(np.float64))
        return 0.5 * (np.square(a).sum() + np.square(b).sum())
    return np.square(a).sum()


@pytest.mark.parametrize("lib", ["F", "D", "DF"])
def test_every_real_complex_field_entry_point(qla, lib):
    man = qla.manifest()
    L = qla.lib()
    rng = np.random.default_rng(600 + len(lib))
    n, ns = 97, 101
    bad, count, approx, approx_same = [], 0, 0, 0.0
    for j, e in enumerate(x for x in man if x["pc"] == lib and x["family"] in ("cfield", "rfield", "sglobal",
                                                                             "convert")):
        ins, idx, gang, want, mode = T.fd_case(e, rng, n, ns)
        keep = []
        args, r_d = _dev_args(e, ins, idx, gang, n, keep, host_const=(j % 2 == 0))
        if mode == "reduce":
            r_h = np.zeros_like(want)
            args[0] = T.ptr(r_h)
            getattr(L, e["name"])(*args)
            got = r_h.astype(np.float64)
            w = want.astype(np.float64)
            scale = _scale(e, ins)
            tol = 1e-13 * scale + (4 * np.spacing(np.abs(want)).astype(np.float64) if want.dtype == np.float32 else 0)
            if lib in ("F", "DF") and e.get("spec") == "LD_NORM2":
                tol = tol + 2 * np.finfo(np.float32).eps * scale
            ok = bool(np.all(np.abs(got - w) <= tol))
        else:
            getattr(L, e["name"])(*args)
            got = T.to_host(r_d)
            if mode == "approx":
                ok = T.within_ulps(got, want, 4)
                approx += 1
                approx_same += float(np.mean(got.ravel() == want.ravel()))
            else:
                ok = T.bits_equal(got, want)
        count += 1
        if not ok:
            bad.append(e["name"])
    qla.check(f"{lib} fields")
    if approx:
        print(f"{lib}: transcendental results bit-identical to the host libm: {approx_same / approx:.4f}")
    assert count >= (64 if lib == "DF" else 900)
    assert not bad, f"{len(bad)} mismatches, e.g. {bad[:10]}"
