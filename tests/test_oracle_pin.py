"""Pins the oracle (oracle/liboracle.so, the CPU restatement) to the reference:

1. against the golden vectors in tests/golden/ (outputs of the reference
   library itself, written by tests/golden/make_golden.py) -- always runs;
2. against the reference library directly on larger seeded inputs, when
   oracle/_ref/libqla_ref.so has been built here.

Linear ops and the reference-order reductions must be bit-identical."""
import ctypes
import os
import re

import numpy as np
import pytest

import qla_testlib as T

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NC = {"V": 3, "H": 6, "D": 12, "M": 9}
NCOL = {"V": 1, "H": 2, "D": 4, "M": 3}


def load(pc):
    z = np.load(os.path.join(GOLDEN, f"qla_{pc.lower()}_golden.npz"))
    ins = {k[4:]: z[k] for k in z.files if k.startswith("in__")}
    outs = {k[5:]: z[k] for k in z.files if k.startswith("out__")}
    return ins, outs


def replay(pc, name, ins):
    """Recompute one golden entry with the oracle."""
    n = len(ins["gang"])
    dt = ins["V"].dtype
    key, *extra = name.split("|")
    m = re.match(r"QLA_(F3|D3|DF3)_([VHDM])_([vx])(eq|peq|meq|eqm)_(p?Ma?)_times_(p?\w+)$", key)
    if m:
        _, dest, var, eq, s1, s2 = m.groups()
        r = (ins["r0" + dest] if dest != "M" else ins["r0M"]).copy()
        bsrc = ins["M2"] if dest == "M" else ins[dest]
        T.ora_lmult(r, ins["M"], bsrc, n, NCOL[dest], eq, adja=int(s1.endswith("a")),
                    adjb=int(s2.endswith("a")), idx_a=ins["idx"] if s1.startswith("p") else None,
                    idx_b=ins["idx"][::-1].copy() if s2.startswith("p") else None,
                    gang=ins["gang"] if var == "x" else None)
        return r
    m = re.match(r"QLA_(F3|D3)_H_([vx])(eq|peq|meq|eqm)_spproj_(p?)D$", key)
    if m:
        _, var, eq, p = m.groups()
        mu, sign = int(extra[0]), int(extra[1])
        r = ins["r0H"].copy()
        T.ora_spproj(r, ins["D"], n, mu, sign, eq, idx_a=ins["idx"] if p else None,
                     gang=ins["gang"] if var == "x" else None)
        return r
    m = re.match(r"QLA_(F3|D3)_P_v(eq|peq|meq|eqm)_(p?)(M|P)(a?)_times_(p?)(M|P)(a?)$", key)
    if m:
        _, eq, _, ta, ca, pb, tb, cb = m.groups()
        kind = {"MP": "MP", "PM": "PM", "PP": "PP"}[ta + tb]
        r = ins["r0P"].copy()
        a = ins["M"] if ta == "M" else ins["P1"]
        b = ins["M"] if tb == "M" else (ins["P2"] if ta == "P" else ins["P1"])
        return T.ora_prop(kind, r, a, b, n, eq, ca=int(bool(ca)), cb=int(bool(cb)), idx_b=ins["idx"] if pb else None)
    m = re.match(r"QLA_(F3|D3)_M_veq_spintrace_P$", key)
    if m:
        r = ins["r0M"].copy()
        return T.ora_prop("TRACE", r, ins["P1"], None, n, "eq")
    m = re.match(r"QLA_(F3|D3)_V_v(eq|peq|meq|eqm)_n(p?)M(a?)_times_n(p?)V$", key)
    if m:
        _, eq, pa, adj, pb = m.groups()
        nd = 4
        r = ins["r0V"].copy()
        return T.ora_multi(r, [ins[f"nm_M{d}"] for d in range(nd)], [ins[f"nm_V{d}"] for d in range(nd)], n, eq,
                           adja=int(bool(adj)), idx_a=ins["idx"] if pa else None,
                           idx_b=ins["idx"][::-1].copy() if pb else None)
    m = re.match(r"QLA_(F3|D3)_(H|D)_v(eq|peq|meq|eqm)_(spproj|sprecon)_(M|Ma)_times_(p?)(D|H)$", key)
    if m:
        _, dest, eq, kind, s1, p, _ = m.groups()
        r = ins["r0" + dest].copy()
        b = ins["D"] if kind == "spproj" else ins["H"]
        return T.ora_hop(r, ins["M"], b, n, int(extra[0]), int(extra[1]), eq, dest, kind, adja=int(s1 == "Ma"),
                         idx_b=ins["idx"] if p else None)
    m = re.match(r"QLA_(F3|D3)_D_v(eq|peq|meq|eqm)_spproj_D$", key)
    if m:
        r = ins["r0D"].copy()
        return T.ora_hop(r, None, ins["D"], n, int(extra[0]), int(extra[1]), m.group(2), "D", "spproj")
    m = re.match(r"QLA_(F3|D3)_D_v(eq|peq|meq|eqm)_sprecon_H$", key)
    if m:
        r = ins["r0D"].copy()
        T.ora_sprecon(r, ins["H"], n, int(extra[0]), int(extra[1]), m.group(2))
        return r
    m = re.match(r"QLA_(F3|D3)_(\w)_v(eq|peq|meq|eqm)_r_times_\w$", key)
    if m:
        dest, eq = m.group(2), m.group(3)
        r = ins["r0" + dest].copy()
        T.ora_rtimes(r, float(ins["scal"][0]), ins[dest if dest != "M" else "M2"], n, NC[dest], eq)
        return r
    m = re.match(r"QLA_(F3|D3|DF3)_r_([vx])eq_norm2_(p?)(\w)$", key)
    if m:
        rpc, var, p, t = m.groups()
        v = T.ora_norm2(ins[t], n, NC[t], idx_a=ins["idx"] if p else None, gang=ins["gang"] if var == "x" else None)
        return np.array([v], dtype=np.float32 if rpc == "F3" else np.float64)
    m = re.match(r"QLA_(F3|D3|DF3)_(c|r)_veq_(re_)?(\w)_dot_\w$", key)
    if m:
        rpc, kind, re_, t = m.groups()
        b = ins["D2"] if t == "D" else ins["M2"] if t == "M" else ins["r0" + t]
        v = T.ora_dot(ins[t], b, n, NC[t])
        odt = np.float32 if rpc == "F3" else np.float64
        return np.array([v.real], dtype=odt) if re_ else np.array([v.real, v.imag], dtype=odt)
    m = re.match(r"QLA_FN_(V|M)_v(eq|peq|meq|eqm)_(M|Ma)_times_(p?)(V|M)$", key)
    if m:
        dest, eq, s1, p2, _ = m.groups()
        nc = int(extra[0])
        if dest == "V":
            r = ins[f"fn{nc}_r0"][:, :2 * nc].copy()
            T.ora_lmult(r, ins[f"fn{nc}_M"], ins[f"fn{nc}_V"], n, 1, eq, nc=nc)
        else:
            r = np.ascontiguousarray(np.tile(ins[f"fn{nc}_r0"][:, :2 * nc], (1, nc)))
            T.ora_lmult(r, ins[f"fn{nc}_M"], ins[f"fn{nc}_M"], n, nc, eq, adja=1, idx_b=ins["idx"], nc=nc)
        return r
    m = re.match(r"QLA_FN_(H|D)_v(eq|peq|meq|eqm)_(spproj|sprecon)_(D|H)$", key)
    if m:
        _, eq, which, _ = m.groups()
        nc, mu = int(extra[0]), int(extra[1])
        if which == "spproj":
            r = ins[f"fn{nc}_r0"][:, :4 * nc].copy()
            T.ora_spproj(r, ins[f"fn{nc}_D"], n, mu, -1, eq, nc=nc)
        else:
            r = ins[f"fn{nc}_r0"][:, :8 * nc].copy()
            T.ora_sprecon(r, ins[f"fn{nc}_H"], n, mu, 1, eq, nc=nc)
        return r
    m = re.match(r"QLA_(FN|DFN)_(r|c)_veq_(norm2_D|V_dot_V)$", key)
    if m:
        rpc, kind, what = m.groups()
        nc = int(extra[0])
        odt = np.float32 if rpc == "FN" else np.float64
        if kind == "r":
            return np.array([T.ora_norm2(ins[f"fn{nc}_D"], n, 4 * nc)], dtype=odt)
        v = T.ora_dot(ins[f"fn{nc}_V"], ins[f"fn{nc}_Vrev"], n, nc)
        return np.array([v.real, v.imag], dtype=odt)
    m = re.match(r"QLA_(F3|D3|FN|DN)_(M|C)_veq_(exp|sqrt|inverse|det)_M$", key)
    if m:
        pcx, _, fname = m.group(1), m.group(2), m.group(3)
        src = extra[0]
        nc = 3 if pcx in ("F3", "D3") else int(src[3])
        return T.ora_mfunc(ins[src], n, fname, nc=nc)
    m = re.match(r"QLA_(F3|D3|FN|DN)_(M|V)_veq_(invsqrt|log|expA|expTA|sqrtPH|invsqrtPH|eigenvals|eigenvalsH)_M$", key)
    if m:
        src = extra[0]
        nc = 3 if m.group(1) in ("F3", "D3") else int(src[3])
        return T.ora_mfunc(ins[src], n, m.group(3), nc=nc)
    m = re.match(r"QLA_(F3|D3)_(V|M)_veq_M_inverse_(V|M)$", key)
    if m:
        return T.ora_minv(ins[extra[0]], ins[extra[1]], n, 1 if m.group(2) == "V" else 3)
    raise KeyError(name)


@pytest.mark.parametrize("pc", ["F3", "D3"])
def test_oracle_matches_reference_golden_vectors(pc):
    ins, outs = load(pc)
    assert len(outs) > 300
    bad = []
    for name, want in outs.items():
        got = replay(pc, name, ins)
        if not T.bits_equal(got, want):
            bad.append(name)
    assert not bad, f"{len(bad)} golden mismatches, e.g. {bad[:5]}"


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref/libqla_ref.so not built")
@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64)])
def test_oracle_matches_reference_library_large(pc, dt):
    """Direct comparison on 20,000 sites (OMP_NUM_THREADS is irrelevant for the
    linear ops; the reductions are compared to the reference's own rounding)."""
    rng = np.random.default_rng(77)
    n = 20000
    R = T.ref()
    a = T.haar_su3(rng, n, dt)
    for dest in ("V", "H", "D", "M"):
        b = T.gaussian_field(rng, n, NC[dest], dt)
        r0 = T.gaussian_field(rng, n, NC[dest], dt)
        for eq in T.EQOPS:
            for s1 in ("M", "Ma"):
                rr = r0.copy()
                getattr(R, f"QLA_{pc}_{dest}_v{eq}_{s1}_times_{dest}")(T.ptr(rr), T.ptr(a), T.ptr(b), n)
                ro = r0.copy()
                T.ora_lmult(ro, a, b, n, NCOL[dest], eq, adja=int(s1 == "Ma"))
                assert T.bits_equal(rr, ro), (dest, eq, s1)
    d = T.gaussian_field(rng, n, 12, dt)
    out = np.zeros(1, dtype=np.float64)
    fn = getattr(R, f"QLA_{'DF3' if pc == 'F3' else 'D3'}_r_veq_norm2_D")
    fn(T.ptr(out), T.ptr(d), n)
    ref_v = out[0]
    ora_v = T.ora_norm2(d, n, 12)
    assert abs(ref_v - ora_v) <= 1e-12 * ref_v


def test_tolerance_rule_matches_reference_harness():
    """test/src/compare.h:10-25: fail only when abs > 16 eps AND rel > 10 eps."""
    eps = np.finfo(np.float32).eps
    ok, _ = T.qla_close([1.0], [1.0 + 8 * eps], np.float32)
    assert ok
    ok, nbad = T.qla_close([100.0], [100.0 * (1 + 20 * eps)], np.float32)
    assert not ok and nbad == 1
    ok, _ = T.qla_close([1e-9], [2e-9], np.float32)  # tiny absolute difference passes
    assert ok


def test_oracle_detects_a_planted_mistake():
    """A mistake planted in the oracle's input (a flipped sign in one matrix
    element) must be caught by the golden comparison."""
    ins, outs = load("F3")
    ins = dict(ins)
    m = ins["M"].copy()
    m[3, 5] = -m[3, 5]
    ins["M"] = m
    name = "QLA_F3_V_veq_M_times_V"
    assert not T.bits_equal(replay("F3", name, ins), outs[name])


def test_int_oracle_matches_reference_golden_vectors():
    """All 238 QLA_I_ v/x entry points of the reference integer library."""
    z = np.load(os.path.join(GOLDEN, "qla_int_golden.npz"))
    ins = {k[4:]: z[k] for k in z.files if k.startswith("in__")}
    outs = {k[5:]: z[k] for k in z.files if k.startswith("out__")}
    assert len(outs) == 238
    bad = [nm for nm, w in outs.items() if not np.array_equal(T.ora_int(nm, ins, len(ins["r0"])), w)]
    assert not bad, bad[:5]


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref (reference headers) not built")
def test_prototypes_match_reference_headers():
    """Every generated entry point that the reference also generates has the
    reference's parameter list (types and order); the rest are the documented
    per-operand index (`xX`) forms and this library's own `qlagpu_` additions."""
    import qla_b200
    ref = {}
    nargs_fn = {}
    for h in ("qla_fn.h", "qla_dfn.h", "qla_dn.h"):
        txt = open(os.path.join(os.path.dirname(T.REF_SO), "gen", "include", h)).read()
        for m in re.finditer(r"void (QLA_(?:D?FN|DN|FDN)_\w+) \((.*?)\);", txt):
            # VLA record types: compare the parameter count (the first is int nc)
            nargs_fn[m.group(1)] = len(re.findall(r"\(\s*\*|\bint\b|QLA_[FD]_(?:Real|Complex)|\bQLA_Int\b|\bQLA_RandomState\b", m.group(2)))
    for h in ("qla_f3.h", "qla_d3.h", "qla_df3.h", "qla_int.h", "qla_f.h", "qla_d.h", "qla_df.h", "qla_f2.h",
              "qla_d2.h", "qla_df2.h"):
        txt = open(os.path.join(os.path.dirname(T.REF_SO), "gen", "include", h)).read()
        for m in re.finditer(r"void (QLA_\w+) \((.*?)\);", txt):
            params = [p.replace("QLA_RESTRICT", "").strip() for p in m.group(2).split(",")]
            # drop the trailing parameter name, keep the type without blanks
            ref[m.group(1)] = [re.match(r"^(.*?)\w+$", p).group(1).replace(" ", "") for p in params]
    extra = []
    for e in qla_b200.manifest():
        if e["name"] in nargs_fn:
            assert len(e["params"]) == nargs_fn[e["name"]], (e["name"], e["params"], nargs_fn[e["name"]])
            continue
        if e["name"].startswith("qlagpu_"):
            continue
        if e["name"] not in ref:
            extra.append(e["name"])
            continue
        ours = [t.replace(" ", "") for t in e["ctypes"]]
        assert ours == ref[e["name"]], (e["name"], ours, ref[e["name"]])
    assert all(re.search(r"_x[VHDMI]$", nm) for nm in extra), [nm for nm in extra if not re.search(r"_x[VHDMI]$", nm)][:5]


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref/libqla_ref.so not built")
@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64)])
def test_oracle_matrix_functions_match_reference_library(pc, dt):
    """Every matrix function and a^-1 b of the code templates, bit for bit,
    on 3,000 sites per input class (closed forms, Newton and Pade paths)."""
    rng = np.random.default_rng(79)
    n = 3000
    R = T.ref()
    ah, _ = T.antihermitian_exp_inputs(rng, n, dt)
    aht = T.from_complex(T.to_complex(ah.astype(np.float64)) + 1j * rng.uniform(-1, 1, n)[:, None, None] * np.eye(3),
                         dt)
    pos = T.positive_hermitian_inputs(rng, n, dt)
    gen = (T.gaussian_field(rng, n, 9, dt) * 0.8).astype(dt)
    herm = T.hermitian_inputs(rng, n, dt)
    cases = [("exp", ah), ("exp", gen), ("sqrt", pos), ("inverse", gen), ("det", gen), ("expTA", ah), ("expA", aht),
             ("log", pos), ("log", gen), ("invsqrt", pos), ("sqrtPH", pos), ("invsqrtPH", pos),
             ("eigenvalsH", herm), ("eigenvals", gen)]
    for fname, a in cases:
        dest = "C" if fname == "det" else "V" if fname.startswith("eigen") else "M"
        nout = {"C": 1, "V": 3, "M": 9}[dest]
        rr = np.zeros((n, 2 * nout), dt)
        getattr(R, f"QLA_{pc}_{dest}_veq_{fname}_M")(T.ptr(rr), T.ptr(a), n)
        assert T.bits_equal(rr, T.ora_mfunc(a, n, fname)), fname
    for dest, nb in (("V", 1), ("M", 3)):
        b = T.gaussian_field(rng, n, 3 * nb, dt)
        rr = np.zeros((n, 6 * nb), dt)
        getattr(R, f"QLA_{pc}_{dest}_veq_M_inverse_{dest}")(T.ptr(rr), T.ptr(gen), T.ptr(b), n)
        assert T.bits_equal(rr, T.ora_minv(gen, b, n, nb)), dest


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref/libqla_ref.so not built")
@pytest.mark.parametrize("pc,dt", [("FN", np.float32), ("DN", np.float64)])
def test_oracle_n_colour_matrix_functions_match_reference_library(pc, dt):
    """The N-colour build's generic paths (Newton invsqrt, log, a^-1 b, and
    the Hessenberg + double-shift QR eigenvalues) at nc = 4 and 8, bit for bit."""
    rng = np.random.default_rng(80)
    n = 1000
    R = T.ref()
    for nc in (4, 8):
        g = rng.standard_normal((n, 2 * nc * nc)).astype(dt)
        pos = T.positive_hermitian_inputs(rng, n, dt, nc=nc)
        herm = T.hermitian_inputs(rng, n, dt, nc=nc)
        for fname, a in (("invsqrt", pos), ("log", pos), ("eigenvals", g), ("eigenvals", herm),
                         ("eigenvalsH", herm), ("eigenvalsH", pos)):
            dest = "V" if fname.startswith("eigen") else "M"
            rr = np.zeros((n, 2 * nc * (1 if dest == "V" else nc)), dt)
            getattr(R, f"QLA_{pc}_{dest}_veq_{fname}_M")(nc, T.ptr(rr), T.ptr(a), n)
            assert T.bits_equal(rr, T.ora_mfunc(a, n, fname, nc=nc)), (nc, fname)
        for dest, nb in (("V", 1), ("M", nc)):
            b = rng.standard_normal((n, 2 * nc * nb)).astype(dt)
            rr = np.zeros((n, 2 * nc * nb), dt)
            getattr(R, f"QLA_{pc}_{dest}_veq_M_inverse_{dest}")(nc, T.ptr(rr), T.ptr(g), T.ptr(b), n)
            assert T.bits_equal(rr, T.ora_minv(g, b, n, nb, nc=nc)), (nc, dest)


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref/libqla_ref.so not built")
@pytest.mark.parametrize("pc,dt", [("F2", np.float32), ("D2", np.float64), ("FN", np.float32), ("DN", np.float64)])
def test_oracle_two_colour_matrix_functions_match_reference_library(pc, dt):
    """The templates' two-colour closed forms (the QLA_F2_/QLA_D2_ builds, and
    the N-colour builds at nc = 2), every matrix function and a^-1 b, bit for
    bit on 3,000 sites per input class, including singular and zero inputs
    of the branches that test for them (det = 0, trace = 0)."""
    rng = np.random.default_rng(81)
    n, nc = 3000, 2
    R = T.ref()
    lead = [nc] if pc in ("FN", "DN") else []
    gen = (rng.standard_normal((n, 8)) * 0.7).astype(dt)
    z = T.to_complex(gen.astype(np.float64), nc)
    ah = T.from_complex(0.5 * (z - np.conj(np.transpose(z, (0, 2, 1)))), dt)
    aht = T.from_complex(T.to_complex(ah.astype(np.float64), nc) + 1j * rng.uniform(-1, 1, n)[:, None, None] * np.eye(2),
                         dt)
    pos = T.positive_hermitian_inputs(rng, n, dt, nc=nc)
    herm = T.hermitian_inputs(rng, n, dt, nc=nc)
    # rank-one and zero matrices (det = 0), scalar multiples of 1 (s^2 - det = 0)
    u = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
    rank1 = np.einsum("ni,nj->nij", u, np.conj(u))
    rank1[::7] = 0
    psd1 = T.from_complex(rank1, dt)
    scal = T.from_complex((rng.uniform(0.5, 2, n) + 1j * rng.uniform(-1, 1, n))[:, None, None] * np.eye(2), dt)
    cases = [("exp", gen), ("exp", ah), ("exp", scal), ("sqrt", pos), ("sqrt", gen), ("sqrt", psd1),
             ("invsqrt", pos), ("invsqrt", gen), ("inverse", gen), ("det", gen), ("det", psd1),
             ("log", pos), ("log", gen), ("log", scal), ("expA", aht), ("expA", ah), ("expTA", ah),
             ("sqrtPH", pos), ("sqrtPH", psd1), ("invsqrtPH", pos), ("eigenvals", gen), ("eigenvals", psd1),
             ("eigenvalsH", herm), ("eigenvalsH", psd1)]
    for fname, a in cases:
        dest = "C" if fname == "det" else "V" if fname.startswith("eigen") else "M"
        nout = {"C": 1, "V": 2, "M": 4}[dest]
        rr = np.zeros((n, 2 * nout), dt)
        getattr(R, f"QLA_{pc}_{dest}_veq_{fname}_M")(*(lead + [T.ptr(rr), T.ptr(a), n]))
        assert T.bits_equal(rr, T.ora_mfunc(a, n, fname, nc=nc)), (pc, fname)
    for dest, nb in (("V", 1), ("M", 2)):
        b = T.gaussian_field(rng, n, 2 * nb, dt)
        rr = np.zeros((n, 4 * nb), dt)
        getattr(R, f"QLA_{pc}_{dest}_veq_M_inverse_{dest}")(*(lead + [T.ptr(rr), T.ptr(gen), T.ptr(b), n]))
        assert T.bits_equal(rr, T.ora_minv(gen, b, n, nb, nc=nc)), (pc, dest)


def _ref_args(e, ins, idx, gang, n, r, ints=None, nc=3):
    """Host arguments of manifest entry e for the reference library."""
    args, keep = [], []
    for t, name in zip(e["ctypes"], e["params"]):
        if name == "n":
            args.append(len(gang) if gang is not None else n)
        elif name == "index":
            args.append(T.ptr(gang))
        elif name == "r":
            args.append(T.ptr(r))
        elif t == "int":
            args.append(ints[name])
        else:
            letter, is_ptr, arr = ins[name]
            if is_ptr:
                rec = T.rec_bytes(letter, arr.dtype, nc)
                pa = (ctypes.c_void_p * len(idx[name]))(*[arr.ctypes.data + int(j) * rec for j in idx[name]])
                keep.append(pa)
                args.append(pa)
            else:
                args.append(T.ptr(arr))
    return args, keep


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref/libqla_ref.so not built")
@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64)])
def test_oracle_elementwise_families_match_reference_library(pc, dt):
    """Every generated element-wise, site-local dot and outer-product entry
    point: the oracle restatement against the reference library, bit for bit
    (all eqops, pointer and gang forms; 13 destination sites, 17 sources)."""
    import json
    man = json.load(open(os.path.join(os.path.dirname(T.ORACLE_SO), "..", "qla_b200", "gen", "api_manifest.json")))
    R = T.ref()
    rng = np.random.default_rng(101)
    n, ns = 13, 17
    bad, count = [], 0
    for e in man:
        if e["pc"] != pc or not (e["family"].startswith("ewise") or e["family"] == "ldot"):
            continue
        ins, idx, gang = T.ewise_inputs(e, rng, dt, n, ns)
        want = T.ewise_oracle(e, ins, idx, gang, n)
        r = ins["r"][2].copy()
        args, keep = _ref_args(e, ins, idx, gang, n, r)
        getattr(R, e["name"])(*args)
        count += 1
        if not T.bits_equal(r, want):
            bad.append(e["name"])
    assert count > 1800
    assert not bad, f"{len(bad)} mismatches, e.g. {bad[:8]}"


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref/libqla_ref.so not built")
@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64)])
def test_oracle_sitefield_families_match_reference_library(pc, dt):
    """Fills, copymask, components, gamma multiplication (all 16 mu for D and
    both sides of P), traces and the antihermitian part: the oracle against
    the reference library, bit for bit, every generated entry point."""
    import json
    man = json.load(open(os.path.join(os.path.dirname(T.ORACLE_SO), "..", "qla_b200", "gen", "api_manifest.json")))
    R = T.ref()
    rng = np.random.default_rng(111)
    n, ns = 13, 17
    bad, count = [], 0
    for e in man:
        if e["pc"] != pc or e["family"] not in T.SF_FAMILIES:
            continue
        reps = 16 if e["family"] == "gamma" else 1
        for rep in range(reps):
            ins, idx, gang, ints = T.sitefield_inputs(e, rng, dt, n, ns)
            if "mu" in ints:
                ints["mu"] = rep
            want = T.sitefield_oracle(e, ins, idx, gang, n, ints)
            r = ins["r"][2].copy()
            args, keep = _ref_args(e, ins, idx, gang, n, r, ints)
            getattr(R, e["name"])(*args)
            count += 1
            if not T.bits_equal(r, want):
                bad.append((e["name"], ints))
    assert count > 300
    assert not bad, f"{len(bad)} mismatches, e.g. {bad[:8]}"


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref/libqla_ref.so not built")
@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64), ("DF3", np.float32)])
def test_oracle_global_p_reductions_and_sums_match_reference_library(pc, dt):
    """Global reductions of P, Ma.M and Pa.P and the global sums: the oracle
    (reference summation order) against the reference library run on one
    OpenMP thread (its sequential order), bit for bit."""
    import json
    man = json.load(open(os.path.join(os.path.dirname(T.ORACLE_SO), "..", "qla_b200", "gen", "api_manifest.json")))
    R = T.ref()
    rng = np.random.default_rng(112)
    n, ns = 13, 17
    bad, count = [], 0
    for e in man:
        if e["pc"] != pc or e["family"] not in ("gred", "gsum"):
            continue
        ins, idx, gang, _ = T.sitefield_inputs(e, rng, dt, n, ns)
        if e["family"] == "gred":
            out = T.gred_oracle(e, ins, idx, gang, n)
            odt = np.float64 if e.get("out") == "double" else dt
            want = out[:1].astype(odt) if e["dest"] == "r" else out.astype(odt)
        else:
            want = T.gsum_oracle(e, ins, idx, gang, n)
        r = np.zeros_like(want)
        args, keep = _ref_args(e, ins, idx, gang, n, r)
        with T.ref_one_thread():
            getattr(R, e["name"])(*args)
        count += 1
        if not T.bits_equal(r, want):
            bad.append(e["name"])
    assert count == 56
    assert not bad, f"{len(bad)} mismatches, e.g. {bad[:8]}"


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref/libqla_ref.so not built")
def test_oracle_precision_conversions_match_reference_library():
    """QLA_DF3_X_*eq_X (float to double) and QLA_FD3_X_*eq_X (double to
    float): the oracle against the reference library, bit for bit."""
    import json
    man = json.load(open(os.path.join(os.path.dirname(T.ORACLE_SO), "..", "qla_b200", "gen", "api_manifest.json")))
    R = T.ref()
    rng = np.random.default_rng(113)
    n, ns = 13, 17
    bad, count = [], 0
    for e in man:
        if e["family"] != "convert" or e["pc"] != "DF3":
            continue
        ins, idx, gang = T.convert_inputs(e, rng, n, ns)
        want = T.convert_oracle(e, ins, idx, gang, n)
        r = ins["r"][2].copy()
        args, keep = _ref_args(e, ins, idx, gang, n, r)
        getattr(R, e["name"])(*args)
        count += 1
        if not T.bits_equal(r, want):
            bad.append(e["name"])
    assert count == 40
    assert not bad, f"{len(bad)} mismatches, e.g. {bad[:8]}"


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref/libqla_ref.so not built")
@pytest.mark.parametrize("lib", ["FN", "DN", "DFN", "F2", "D2", "DF2"])
def test_oracle_ncolor_families_match_reference_library(lib):
    """The element-wise, site-local product, fill / component / gamma /
    trace families, global P / adjoint-form reductions, sums and conversions
    of the N-colour libraries at nc = 2 and 5: the oracle against the
    reference library, bit for bit, every entry point (the reductions and
    sums with the library on one OpenMP thread)."""
    import qla_b200
    man = qla_b200.manifest()
    byname = {e["name"]: e for e in man}
    R = T.ref()
    rng = np.random.default_rng(114)
    n, ns = 7, 9
    bad, count = [], 0
    for e in man:
        if e["pc"] != lib or e["family"] not in T.NCOLOR_FAMILIES:
            continue
        twin = byname[T.fixed_colour_twin(e["name"])]
        two = lib.endswith("2")
        for nc in ((2,) if two else (2, 5)):
            (ins, idx, gang, ints), want, kind = T.ncolor_case(twin, rng, n, ns, nc)
            if "mu" in ints:
                ints["mu"] = count % 16
                want = T.sitefield_oracle(twin, ins, idx, gang, n, ints, nc=nc)
            r = np.zeros_like(want) if kind in ("gred", "gsum") else ins["r"][2].copy()
            args, keep = _ref_args(twin, ins, idx, gang, n, r, ints, nc=nc)
            with T.ref_one_thread():
                getattr(R, e["name"])(*(([] if two else [nc]) + args))
            count += 1
            if not T.bits_equal(r, want):
                bad.append((e["name"], nc))
    assert count > ((75 if two else 150) if lib.startswith("DF") else (1000 if two else 2000))
    assert not bad, f"{len(bad)} mismatches, e.g. {bad[:8]}"


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref/libqla_ref.so not built")
@pytest.mark.parametrize("lib,dt", [("FN", np.float32), ("DN", np.float64)])
def test_oracle_ncolor_hop_terms_match_reference_library(lib, dt):
    """The fused hop terms of the N-colour libraries (spproj / sprecon with a
    colour-matrix multiply, every eqop, M and Ma, every mu and sign) at
    nc = 2 and 4: the oracle composition against the reference, bit for bit."""
    import itertools
    R = T.ref()
    rng = np.random.default_rng(115)
    n = 11
    for nc in (2, 4):
        a = rng.standard_normal((n, 2 * nc * nc)).astype(dt)
        d = rng.standard_normal((n, 8 * nc)).astype(dt)
        h = rng.standard_normal((n, 4 * nc)).astype(dt)
        r0 = {"H": rng.standard_normal((n, 4 * nc)).astype(dt), "D": rng.standard_normal((n, 8 * nc)).astype(dt)}
        for (dest, kind), eq, s1, (mu, sign) in itertools.product(
                [("H", "spproj"), ("D", "spproj"), ("D", "sprecon")], T.EQOPS, ["M", "Ma"],
                [(0, 1), (1, -1), (2, 1), (3, -1), (4, 1), (4, -1)]):
            src, b = ("D", d) if kind == "spproj" else ("H", h)
            rr = r0[dest].copy()
            getattr(R, f"QLA_{lib}_{dest}_v{eq}_{kind}_{s1}_times_{src}")(nc, T.ptr(rr), T.ptr(a), T.ptr(b), mu, sign,
                                                                          n)
            want = r0[dest].copy()
            T.ora_hop(want, a, b, n, mu, sign, eq, dest, kind, adja=int(s1 == "Ma"), nc=nc)
            assert T.bits_equal(rr, want), (lib, nc, dest, kind, eq, s1, mu, sign)


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref/libqla_ref.so not built")
@pytest.mark.parametrize("lib,dt", [("FN", np.float32), ("DN", np.float64)])
def test_oracle_ncolor_propagator_products_match_reference_library(lib, dt):
    """Every N-colour DiracPropagator product and spin trace entry point at
    nc = 2 and 4: the oracle against the reference library, bit for bit."""
    import qla_b200
    R = T.ref()
    rng = np.random.default_rng(116)
    n, ns = 5, 7
    names = [e["name"] for e in qla_b200.manifest() if e["pc"] == lib and e["family"] == "prop"]
    assert len(names) == 388
    for nc in (2, 4):
        data, cases = T.prop_cases(lib, names, nc, dt, rng, n, ns)
        cbytes = 2 * np.dtype(dt).itemsize
        keep = []

        def host_ptrs(key, idx):
            rec = cbytes * (nc * nc if key == "M" else 16 * nc * nc)
            arr = data[key]
            pa = (ctypes.c_void_p * len(idx))(*[arr.ctypes.data + int(j) * rec for j in idx])
            keep.append(pa)
            return pa

        bad = []
        for name, spec, want in cases:
            r = spec["r0"].copy()
            ka, pa = spec["a"]
            args = [nc, T.ptr(r), host_ptrs(ka, data["ia"]) if pa else T.ptr(data[ka])]
            if spec["b"] is not None:
                kb, pb = spec["b"]
                args.append(host_ptrs(kb, data["ib"]) if pb else T.ptr(data[kb]))
            if spec["var"] == "x":
                args.append(T.ptr(data["gang"]))
            getattr(R, name)(*args, n)
            if not T.bits_equal(r, want):
                bad.append((name, nc))
        assert not bad, f"{len(bad)} mismatches, e.g. {bad[:6]}"


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref/libqla_ref.so not built")
@pytest.mark.parametrize("lib,dt", [("FN", np.float32), ("DN", np.float64)])
def test_oracle_ncolor_multi_direction_sums_match_reference_library(lib, dt):
    """QLA_FN_ / QLA_DN_ V_*_n{p}M{a}_times_n{p}V at nc = 2 and 4 with nd = 3:
    the oracle's per-direction composition against the reference, bit for bit."""
    import itertools
    R = T.ref()
    rng = np.random.default_rng(117)
    n, nd = 9, 3
    for nc in (2, 4):
        ms = [rng.standard_normal((n, 2 * nc * nc)).astype(dt) for _ in range(nd)]
        vs = [rng.standard_normal((n, 2 * nc)).astype(dt) for _ in range(nd)]
        r0 = rng.standard_normal((n, 2 * nc)).astype(dt)
        ta = (ctypes.c_void_p * nd)(*[m.ctypes.data for m in ms])
        tb = (ctypes.c_void_p * nd)(*[v.ctypes.data for v in vs])
        for eq, s1 in itertools.product(T.EQOPS, ["nM", "nMa"]):
            rr = r0.copy()
            getattr(R, f"QLA_{lib}_V_v{eq}_{s1}_times_nV")(nc, T.ptr(rr), ta, tb, n, nd)
            want = r0.copy()
            T.ora_multi(want, ms, vs, n, eq, adja=int(s1 == "nMa"), nc=nc)
            assert T.bits_equal(rr, want), (lib, nc, eq, s1)


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref/libqla_ref.so not built")
@pytest.mark.parametrize("milc", [0, 1])
def test_oracle_random_generator_matches_reference_library(milc):
    """QLA_seed_random, QLA_random and QLA_gaussian (Box-Muller, and MILC's
    polar method with the switch set): the oracle against the reference's
    lib/random, value and state bit for bit over many draws."""
    R = T.ref()
    O = T.oracle()
    R.QLA_random.restype = ctypes.c_float
    R.QLA_gaussian.restype = ctypes.c_float
    O.ora_rng_uniform.restype = ctypes.c_float
    O.ora_rng_gaussian.restype = ctypes.c_float
    flag = ctypes.c_int.in_dll(R, "QLA_use_milc_gaussian")
    flag.value = milc
    try:
        rng = np.random.default_rng(118)
        for _ in range(40):
            seed, index = int(rng.integers(-2**31, 2**31 - 1)), int(rng.integers(0, 1 << 22))
            a = np.zeros(11, np.uint32)
            b = np.zeros(11, np.uint32)
            R.QLA_seed_random(T.ptr(a), seed, index)
            O.ora_rng_seed(T.ptr(b), seed, index)
            assert T.bits_equal(a, b)
            for j in range(300):
                if j % 3 == 0:
                    x, y = R.QLA_random(T.ptr(a)), O.ora_rng_uniform(T.ptr(b))
                else:
                    x, y = R.QLA_gaussian(T.ptr(a)), O.ora_rng_gaussian(T.ptr(b), milc)
                assert np.float32(x).tobytes() == np.float32(y).tobytes()
            assert T.bits_equal(a, b)
    finally:
        flag.value = 0


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref/libqla_ref.so not built")
@pytest.mark.parametrize("milc", [0, 1])
def test_oracle_random_fills_match_reference_library(milc):
    """Every uniform / gaussian fill, seeding and state copy entry point of
    the F3, D3, F, D, integer and (nc = 2) N-colour libraries: the oracle
    against the reference library, values and states bit for bit."""
    import qla_b200
    man = qla_b200.manifest()
    byname = {e["name"]: e for e in man}
    R = T.ref()
    flag = ctypes.c_int.in_dll(R, "QLA_use_milc_gaussian")
    flag.value = milc
    rng = np.random.default_rng(119)
    n, ns = 7, 9
    bad, count = [], 0
    try:
        for e in man:
            if e["family"] != "random":
                continue
            nc, lead = 3, []
            twin = e
            if e["pc"] in ("FN", "DN"):
                twin, nc, lead = byname[T.fixed_colour_twin(e["name"])], 2, [2]
            elif e["pc"] in ("F2", "D2"):
                twin, nc, lead = byname[T.fixed_colour_twin(e["name"])], 2, []
            if milc and twin.get("op") != "gaussian":
                continue
            ins, idx, gang, ints, want_r, want_s = T.random_case(twin, rng, n, ns, nc=nc, milc=milc)
            r = ins["r"][2].copy()
            st = ins["a"][2].copy() if ins["a"][0] == "S" else None
            if st is not None:
                ins = dict(ins, a=("S", ins["a"][1], st))
            args, keep = _ref_args(twin, ins, idx, gang, n, r, ints, nc=nc)
            getattr(R, e["name"])(*(lead + args))
            count += 1
            ok = T.bits_equal(r, want_r) and (want_s is None or T.bits_equal(st, want_s))
            if not ok:
                bad.append(e["name"])
    finally:
        flag.value = 0
    assert count >= (128 if milc else 160)
    assert not bad, f"{len(bad)} mismatches, e.g. {bad[:8]}"


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref/libqla_ref.so not built")
@pytest.mark.parametrize("lib", ["F", "D", "DF"])
def test_oracle_real_complex_field_libraries_match_reference_library(lib):
    """Every entry point of the real / complex / integer field libraries
    (QLA_F_, QLA_D_, QLA_DF_ / QLA_FD_): the oracle against the reference
    library, bit for bit, including the libm functions (the oracle calls the
    same host libm) and the global reductions (library on one OpenMP thread)."""
    import qla_b200
    R = T.ref()
    rng = np.random.default_rng(121)
    n, ns = 11, 13
    bad, count = [], 0
    for e in qla_b200.manifest():
        if e["pc"] != lib or e["family"] not in ("cfield", "rfield", "sglobal", "convert"):
            continue
        ins, idx, gang, want, mode = T.fd_case(e, rng, n, ns)
        r = np.zeros_like(want) if mode == "reduce" else ins["r"][2].copy()
        args, keep = _ref_args(e, ins, idx, gang, n, r)
        with T.ref_one_thread():
            getattr(R, e["name"])(*args)
        count += 1
        if not T.bits_equal(r, want):
            bad.append(e["name"])
    assert count >= (64 if lib == "DF" else 900)
    assert not bad, f"{len(bad)} mismatches, e.g. {bad[:10]}"


@pytest.mark.skipif(not T.ref_available(), reason="oracle/_ref/libqla_ref.so not built")
def test_qla_rng_inputs_match_the_reference_generator():
    """The per-site generator draws used for the config-1 inputs
    (qla_testlib.qla_rng_gaussian) are the reference library's own
    QLA_seed_random / QLA_gaussian deviates."""
    R = T.ref()
    R.QLA_gaussian.restype = ctypes.c_float
    g = T.qla_rng_gaussian(1234, 64, 18)
    for i in (0, 1, 17, 63):
        st = np.zeros(11, np.uint32)
        R.QLA_seed_random(T.ptr(st), 1234, i)
        want = np.array([R.QLA_gaussian(T.ptr(st)) for _ in range(18)], np.float32)
        assert np.array_equal(g[i], want), i
