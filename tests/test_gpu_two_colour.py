"""GPU check of the two-colour libraries (QLA_F2_, QLA_D2_, QLA_DF2_,
QLA_FD2_): every entry point against the N-colour entry point of the same
name at nc = 2, on identical copies of seeded inputs, every buffer compared
bit for bit afterwards (outputs, and state fields that the random fills
update).  The N-colour entry points are tested against the oracle at nc = 2
(tests/test_gpu_ncolor.py, tests/test_gpu_fn.py) and the oracle against the
reference's two-colour libraries (tests/test_oracle_pin.py).  The matrix
functions of both are the templates' two-colour closed forms."""
import ctypes
import re

import numpy as np
import pytest

import qla_testlib as T

pytestmark = pytest.mark.gpu

NE2 = {"ColorVector": 2, "HalfFermion": 4, "DiracFermion": 8, "ColorMatrix": 4, "DiracPropagator": 64}


def _elem(ctype):
    """(numpy dtype, values per record) of a parameter type, or None."""
    m = re.search(r"QLA_(F|D)2_(\w+)", ctype)
    if m:
        return (np.float32 if m.group(1) == "F" else np.float64), 2 * NE2[m.group(2)]
    if "QLA_F_Complex" in ctype:
        return np.float32, 2
    if "QLA_D_Complex" in ctype:
        return np.float64, 2
    if "QLA_F_Real" in ctype:
        return np.float32, 1
    if "QLA_D_Real" in ctype:
        return np.float64, 1
    if "QLA_Int" in ctype:
        return np.int32, 1
    if "QLA_RandomState" in ctype:
        return np.uint32, 11
    return None


def _case(e, rng, n, ns):
    """Host buffers and a builder of the C arguments for entry e."""
    bufs, ints, ptrs = {}, {}, {}
    for t, name in zip(e["ctypes"], e["params"]):
        if name in ("n", "index"):
            continue
        if t == "int":
            ints[name] = {"mu": int(rng.integers(0, 5)) if e["family"] in ("spproj", "sprecon", "hop")
                          else int(rng.integers(0, 16)), "sign": 1 if rng.random() < 0.5 else -1,
                          "i_c": int(rng.integers(0, 2)), "j_c": int(rng.integers(0, 2)), "i_s": 1, "j_s": 3,
                          "seed": 12345, "nd": 3}.get(name, 1)
            continue
        if name == "jb":  # the int32 per-operand index of the xX forms
            bufs[(name, 0)] = rng.integers(0, ns, (ns, 1)).astype(np.int32)
            ptrs[name] = (False, False, 4)
            continue
        dt, per = _elem(t)
        multi = e["family"] == "multi" and name in ("a", "b")
        depth = t.replace(" ", "").count("*")
        count = 3 if multi else 1
        for d in range(count):
            key = (name, d)
            if dt == np.int32:
                arr = rng.integers(-3, 4, (ns, per)).astype(np.int32)
            elif dt == np.uint32:
                arr = rng.integers(0, 2**32, (ns, per), dtype=np.uint64).astype(np.uint32)
            else:
                arr = rng.standard_normal((ns, per)).astype(dt)
            bufs[key] = arr
        # pointer arrays: one level for p forms, two for the multi tables of p forms
        ptrs[name] = (depth - (1 if multi else 0)) >= 2, multi, per * np.dtype(dt).itemsize
    gang = rng.permutation(n)[: n // 2 + 1].astype(np.int32)
    idx = rng.integers(0, ns, ns).astype(np.int32)
    return bufs, ints, ptrs, gang, idx


def _run(L, name, lead, e, bufs, ints, ptrs, gang, idx, n):
    dev = {k: T.to_dev(v) for k, v in bufs.items()}
    keep = []
    args = []
    for t, pname in zip(e["ctypes"], e["params"]):
        if pname == "n":
            # the x forms loop over the entries of the gang index
            args.append(len(gang) if "index" in e["params"] else n)
        elif pname == "index":
            g = T.to_dev(gang)
            keep.append(g)
            args.append(T.ptr_dev(g))
        elif t == "int":
            args.append(ints[pname])
        else:
            is_ptr, multi, rec = ptrs[pname]
            if multi:
                addrs = []
                for d in range(3):
                    base = dev[(pname, d)]
                    if is_ptr:
                        pa = T.ptr_array(base, idx, rec)
                        keep.append(pa)
                        addrs.append(pa.data_ptr())
                    else:
                        addrs.append(base.data_ptr())
                tab = T.to_dev(np.array(addrs, np.int64))
                keep.append(tab)
                args.append(T.ptr_dev(tab))
            elif is_ptr:
                pa = T.ptr_array(dev[(pname, 0)], idx, rec)
                keep.append(pa)
                args.append(T.ptr_dev(pa))
            else:
                args.append(T.ptr_dev(dev[(pname, 0)]))
    fn = getattr(L, name)
    fn.restype = None
    fn(*([ctypes.c_int(a) if isinstance(a, int) else a for a in lead + args]))
    return {k: T.to_host(v) for k, v in dev.items()}


@pytest.mark.parametrize("lib", ["F2", "D2", "DF2"])
def test_two_colour_entry_points_equal_n_colour_at_nc2(qla, lib):
    man = qla.manifest()
    L = qla.lib()
    rng = np.random.default_rng(700 + len(lib))
    n, ns = 29, 31
    bad, count = [], 0
    for e in (x for x in man if x["pc"] == lib):
        m = re.match(r"QLA_(F2|D2|DF2|FD2)_(.*)$", e["name"])
        twin = "QLA_" + {"F2": "FN", "D2": "DN", "DF2": "DFN", "FD2": "FDN"}[m.group(1)] + "_" + m.group(2)
        bufs, ints, ptrs, gang, idx = _case(e, rng, n, ns)
        qla.clear_error()
        got = _run(L, e["name"], [], e, bufs, ints, ptrs, gang, idx, n)
        err2 = qla.last_error()[0]
        qla.clear_error()
        want = _run(L, twin, [2], e, bufs, ints, ptrs, gang, idx, n)
        errn = qla.last_error()[0]
        qla.clear_error()
        count += 1
        same = all(T.bits_equal(got[k], want[k]) for k in got) and (err2 != 0) == (errn != 0)
        if not same:
            bad.append(e["name"])
    assert count >= (170 if lib == "DF2" else 3400)
    assert not bad, f"{len(bad)} differences, e.g. {bad[:8]}"
