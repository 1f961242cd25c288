"""GPU parity of the random-number families through the C-ABI: uniform fills
(R_*_random_S), gaussian fills of every field type (F3, D3, F, D, and the
N-colour libraries at nc = 2 and 4), seeding (S_*_seed_i_I) and state copies
(S_*_S, S_*_S_mask_I), against the oracle (pinned to the reference's
lib/random, tests/test_oracle_pin.py).

Uniform deviates, seeding, copies and every generator state left behind are
bit-exact.  Gaussian deviates are rounded to float from a double computed
with the device's log / cos, which may differ from the host libm in the last
place of the double: each value must be within 1 float ulp of the oracle's,
and at least 99.9% of them bit-identical (the test prints the fraction).
The MILC polar method (QLA_use_milc_gaussian != 0) is tested the same way."""
import ctypes

import numpy as np
import pytest

import qla_testlib as T

pytestmark = pytest.mark.gpu


def _dev_args(e, ins, idx, gang, n, ints, keep, nc):
    args, r_d, s_d = [], None, None
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
            base = T.to_dev(arr)
            keep.append(base)
            if letter == "S":
                s_d = base
            if is_ptr:
                pa = T.ptr_array(base, idx[name], T.rec_bytes(letter, arr.dtype, nc))
                keep.append(pa)
                args.append(T.ptr_dev(pa))
            else:
                args.append(T.ptr_dev(base))
    return args, r_d, s_d


def _ulp_close(got, want):
    g = np.asarray(got, np.float32).ravel().astype(np.float64)
    w = np.asarray(want, np.float32).ravel().astype(np.float64)
    ulp = np.spacing(np.abs(np.asarray(want, np.float32).ravel())).astype(np.float64)
    return np.all(np.abs(g - w) <= ulp), np.mean(g == w) if g.size else 1.0


@pytest.mark.parametrize("milc", [0, 1])
def test_every_random_entry_point(qla, milc):
    man = qla.manifest()
    byname = {e["name"]: e for e in man}
    L = qla.lib()
    flag = ctypes.c_int.in_dll(L, "QLA_use_milc_gaussian")
    flag.value = milc
    rng = np.random.default_rng(500 + milc)
    n, ns = 173, 181
    bad, count, same, total = [], 0, 0.0, 0
    try:
        for e in (x for x in man if x["family"] == "random"):
            ncs = [3]
            twin = e
            if e["pc"] in ("FN", "DN"):
                twin, ncs = byname[T.fixed_colour_twin(e["name"])], [2, 4]
            elif e["pc"] in ("F2", "D2"):
                twin, ncs = byname[T.fixed_colour_twin(e["name"])], [2]
            if milc and twin.get("op") != "gaussian":
                continue
            for nc in ncs:
                ins, idx, gang, ints, want_r, want_s = T.random_case(twin, rng, n, ns, nc=nc, milc=milc)
                keep = []
                args, r_d, s_d = _dev_args(twin, ins, idx, gang, n, ints, keep, nc)
                lead = [nc] if e["pc"] in ("FN", "DN") else []
                getattr(L, e["name"])(*(lead + args))
                count += 1
                got_r = T.to_host(r_d)
                if twin.get("op") == "gaussian":
                    ok, frac = _ulp_close(got_r, want_r)
                    same += frac
                    total += 1
                else:
                    ok = T.bits_equal(got_r, want_r)
                if want_s is not None:
                    ok = ok and T.bits_equal(T.to_host(s_d), want_s)
                if not ok:
                    bad.append((e["name"], nc))
    finally:
        flag.value = 0
    qla.check("random")
    assert qla.lib().qlagpu_device_error(1) == 0
    print(f"gaussian values bit-identical to the oracle: {same / max(total, 1):.6f} (milc={milc})")
    assert count >= (120 if milc else 160)
    assert not bad, f"{len(bad)} mismatches, e.g. {bad[:8]}"
    assert same / max(total, 1) >= 0.999


def test_gaussian_fill_large_field_statistics(qla, cuda):
    """2^20 sites of F3 ColorVectors: the gaussian fill's moments (mean 0,
    variance 1) and the generator states agree with a second fill started
    from copies of the same states (determinism)."""
    rng = np.random.default_rng(502)
    n = 1 << 20
    st = np.zeros((n, 11), np.uint32)
    seeds = np.arange(n, dtype=np.int32)
    L = qla.lib()
    s_d = T.to_dev(st)
    a_d = T.to_dev(seeds)
    L.QLA_S_veq_seed_i_I(T.ptr_dev(s_d), 1234567, T.ptr_dev(a_d), n)
    s2 = cuda.empty_like(s_d)
    L.QLA_S_veq_S(T.ptr_dev(s2), T.ptr_dev(s_d), n)
    r1 = cuda.empty((n, 6), dtype=cuda.float32, device="cuda")
    r2 = cuda.empty((n, 6), dtype=cuda.float32, device="cuda")
    L.QLA_F3_V_veq_gaussian_S(T.ptr_dev(r1), T.ptr_dev(s_d), n)
    L.QLA_F3_V_veq_gaussian_S(T.ptr_dev(r2), T.ptr_dev(s2), n)
    qla.check("large gaussian")
    x = r1.cpu().numpy().astype(np.float64)
    assert T.bits_equal(r1.cpu().numpy(), r2.cpu().numpy())
    assert T.bits_equal(s_d.cpu().numpy(), s2.cpu().numpy())
    assert abs(x.mean()) < 5e-3 and abs(x.var() - 1.0) < 5e-3
    # spot-check 64 sites against the oracle bit for bit in the states
    sel = rng.choice(n, 64, replace=False)
    st0 = np.zeros((n, 11), np.uint32)
    T.oracle().ora_rng_seedfield(T.ptr(st0), 1234567, T.ptr(seeds), n, None, None)
    want = np.zeros((n, 6), np.float32)
    T.oracle().ora_rng_fill_f(6, 1, 0, T.ptr(want), T.ptr(st0), n, None, None)
    assert T.bits_equal(s_d.cpu().numpy()[sel], st0[sel])
    ok, frac = _ulp_close(x[sel].astype(np.float32), want[sel])
    assert ok and frac > 0.99
