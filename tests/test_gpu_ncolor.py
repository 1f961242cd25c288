"""GPU parity of the N-colour element-wise, site-local product, fill /
component / gamma / trace, global reduction, global sum and conversion
families (QLA_FN_, QLA_DN_, QLA_DFN_, QLA_FDN_) through the C-ABI, at
nc = 2, 4 and 5 (any nc is served by the same kernels): every entry point
against the oracle, maps bit for bit, reductions and sums within the
tolerance of tests/test_gpu_sitefield.py.  The oracle is pinned to the
reference's N-colour libraries entry point by entry point
(tests/test_oracle_pin.py::test_oracle_ncolor_families_match_reference_library)."""
import numpy as np
import pytest

import qla_testlib as T

pytestmark = pytest.mark.gpu


def _dev_args(e, ins, idx, gang, n, ints, keep, nc, host_const):
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
                pa = T.ptr_array(base, idx[name], T.rec_bytes(letter, arr.dtype, nc))
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


@pytest.mark.parametrize("lib", ["FN", "DN", "DFN"])
@pytest.mark.parametrize("nc", [2, 4, 5])
def test_every_ncolor_entry_point(qla, cuda, lib, nc):
    import qla_b200
    man = qla_b200.manifest()
    byname = {e["name"]: e for e in man}
    L = qla.lib()
    rng = np.random.default_rng(400 + nc)
    n, ns = 37, 41
    bad, count = [], 0
    for j, e in enumerate(x for x in man if x["pc"] == lib and x["family"] in T.NCOLOR_FAMILIES):
        twin = byname[T.fixed_colour_twin(e["name"])]
        (ins, idx, gang, ints), want, kind = T.ncolor_case(twin, rng, n, ns, nc)
        if "mu" in ints:
            ints["mu"] = j % 16
            want = T.sitefield_oracle(twin, ins, idx, gang, n, ints, nc=nc)
        keep = []
        host_const = twin.get("op") in ("fill", "diagfill") and j % 2 == 0
        args, r_d = _dev_args(twin, ins, idx, gang, n, ints, keep, nc, host_const)
        if kind in ("gred", "gsum"):
            odt = want.dtype
            r_h = np.zeros_like(want)
            args[0] = T.ptr(r_h)
            getattr(L, e["name"])(nc, *args)
            got = r_h.astype(np.float64)
            w = want.astype(np.float64)
            a = ins["a"][2].astype(np.float64)
            if kind == "gsum":
                scale = np.abs(a).sum() + 1e-300
            else:
                scale = np.abs(a).sum() * (np.abs(ins["b"][2]).max() if "b" in ins else np.abs(a).max()) + 1e-300
            tol = 1e-13 * scale + (8 * np.finfo(np.float32).eps * np.abs(w) if odt == np.float32 else 0)
            if ins["a"][2].dtype == np.float32 and twin.get("kind") == "LD_NORM2":
                tol = tol + 2 * np.finfo(np.float32).eps * scale
            ok = bool(np.all(np.abs(got - w) <= tol))
        else:
            getattr(L, e["name"])(nc, *args)
            ok = T.bits_equal(T.to_host(r_d), want)
        count += 1
        if not ok:
            bad.append(e["name"])
    qla.check(f"{lib} nc={nc}")
    assert count > (90 if lib == "DFN" else 2000)
    assert not bad, f"{len(bad)} mismatches, e.g. {bad[:8]}"


def test_ncolor_outside_range_is_refused(qla):
    qla.clear_error()
    qla.lib().QLA_FN_V_veq_zero(0, None, 10)
    code, msg = qla.last_error()
    assert code == 4 and "nc" in msg
    qla.clear_error()
