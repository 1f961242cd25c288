#!/usr/bin/env python3
"""Writes the golden vectors of the QLA hot path by running the REFERENCE
library itself (oracle/_ref/libqla_ref.so, built from the reference's own
generator by oracle/build_ref.sh) on seeded inputs.

QLA ships no golden data (its tests compare the library against itself,
test/src/protocol_tensor_sng.m4, protocol_idx.m4), so these fixtures are the
reference's outputs recorded here.  Run with OMP_NUM_THREADS=1 so the
reductions use the serial summation order:

    OMP_NUM_THREADS=1 python tests/golden/make_golden.py

Output: tests/golden/qla_<pc>_golden.npz  (inputs, index tables, outputs)
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import qla_testlib as T  # noqa: E402

N = 37      # destination sites
NS = 41     # source records (gathers index into these)
EQOPS = ["eq", "peq", "meq", "eqm"]


def build(pc, dt, seed):
    rng = np.random.default_rng(seed)
    R = T.ref()
    P = pc[0]
    ins = {
        "M": T.haar_su3(rng, NS, dt),
        "M2": T.haar_su3(rng, NS, dt),
        "V": T.gaussian_field(rng, NS, 3, dt),
        "H": T.gaussian_field(rng, NS, 6, dt),
        "D": T.gaussian_field(rng, NS, 12, dt),
        "D2": T.gaussian_field(rng, NS, 12, dt),
        "r0V": T.gaussian_field(rng, N, 3, dt),
        "r0H": T.gaussian_field(rng, N, 6, dt),
        "r0D": T.gaussian_field(rng, N, 12, dt),
        "r0M": T.gaussian_field(rng, N, 9, dt),
        "idx": rng.integers(0, NS, N).astype(np.int32),
        "gang": rng.permutation(N).astype(np.int32),
        "scal": np.array([-0.6181], dtype=dt),
    }
    out = {}
    recb = 8 if dt == np.float32 else 16

    def parr(arr, idx, ncplx):
        base = arr.ctypes.data
        return (ctypes.c_void_p * len(idx))(*[base + int(j) * ncplx * recb for j in idx])

    def call(name, *args):
        getattr(R, name)(*args)

    # left multiplication (all eqops, adjoints, pointer and gang variants on V;
    # a representative set on H, D, M)
    for dest, nc in (("V", 3), ("H", 6), ("D", 12), ("M", 9)):
        for eq in EQOPS:
            for s1 in ("M", "Ma", "pM", "pMa"):
                for s2 in (dest, "p" + dest) + (("Ma", "pMa") if dest == "M" else ()):
                    if dest != "V" and eq not in ("eq", "peq"):
                        continue
                    for var in ("v", "x"):
                        name = f"QLA_{pc}_{dest}_{var}{eq}_{s1}_times_{s2}"
                        r = ins["r0" + dest][:N].copy() if dest != "M" else ins["r0M"].copy()
                        a = parr(ins["M"], ins["idx"], 9) if s1.startswith("p") else ins["M"].ctypes.data
                        bsrc = ins["M2"] if dest == "M" else ins[dest]
                        b = parr(bsrc, ins["idx"][::-1].copy(), nc) if s2.startswith("p") else bsrc.ctypes.data
                        args = [ctypes.c_void_p(r.ctypes.data), a if s1.startswith("p") else ctypes.c_void_p(a),
                                b if s2.startswith("p") else ctypes.c_void_p(b)]
                        if var == "x":
                            args.append(ctypes.c_void_p(ins["gang"].ctypes.data))
                        args.append(N)
                        call(name, *args)
                        out[name] = r
    # spin projection / reconstruction, every mu and sign
    for eq in EQOPS:
        for mu in range(6):
            for sign in (1, -1):
                r = ins["r0H"].copy()
                call(f"QLA_{pc}_H_v{eq}_spproj_D", ctypes.c_void_p(r.ctypes.data),
                     ctypes.c_void_p(ins["D"].ctypes.data), mu, sign, N)
                out[f"QLA_{pc}_H_v{eq}_spproj_D|{mu}|{sign}"] = r
                r = ins["r0D"].copy()
                call(f"QLA_{pc}_D_v{eq}_sprecon_H", ctypes.c_void_p(r.ctypes.data),
                     ctypes.c_void_p(ins["H"].ctypes.data), mu, sign, N)
                out[f"QLA_{pc}_D_v{eq}_sprecon_H|{mu}|{sign}"] = r
        r = ins["r0H"].copy()
        call(f"QLA_{pc}_H_x{eq}_spproj_pD", ctypes.c_void_p(r.ctypes.data), parr(ins["D"], ins["idx"], 12), 2, -1,
             ctypes.c_void_p(ins["gang"].ctypes.data), N)
        out[f"QLA_{pc}_H_x{eq}_spproj_pD|2|-1"] = r
    # DiracPropagator products and spin trace
    ins["P1"] = T.gaussian_field(rng, NS, 144, dt)
    ins["P2"] = T.gaussian_field(rng, NS, 144, dt)
    ins["r0P"] = T.gaussian_field(rng, N, 144, dt)
    for name, aa, bb, pb in ((f"QLA_{pc}_P_vpeq_M_times_P", "M", "P1", False),
                             (f"QLA_{pc}_P_veq_Ma_times_pPa", "M", "P1", True),
                             (f"QLA_{pc}_P_vmeq_Pa_times_M", "P1", "M", False),
                             (f"QLA_{pc}_P_veqm_P_times_pMa", "P1", "M", True),
                             (f"QLA_{pc}_P_veq_P_times_P", "P1", "P2", False),
                             (f"QLA_{pc}_P_vpeq_Pa_times_pP", "P1", "P2", True),
                             (f"QLA_{pc}_P_veq_P_times_Pa", "P1", "P2", False)):
        r = ins["r0P"].copy()
        nb = 9 if bb == "M" else 144
        b = parr(ins[bb], ins["idx"], nb) if pb else ctypes.c_void_p(ins[bb].ctypes.data)
        call(name, ctypes.c_void_p(r.ctypes.data), ctypes.c_void_p(ins[aa].ctypes.data), b, N)
        out[name] = r
    r = ins["r0M"].copy()
    call(f"QLA_{pc}_M_veq_spintrace_P", ctypes.c_void_p(r.ctypes.data), ctypes.c_void_p(ins["P1"].ctypes.data), N)
    out[f"QLA_{pc}_M_veq_spintrace_P"] = r
    # multi-direction accumulation, nd = 4 directions (host arrays of fields)
    nd = 4
    ms = [T.haar_su3(rng, NS, dt) for _ in range(nd)]
    vs = [T.gaussian_field(rng, NS, 3, dt) for _ in range(nd)]
    for d in range(nd):
        ins[f"nm_M{d}"], ins[f"nm_V{d}"] = ms[d], vs[d]
    am = (ctypes.c_void_p * nd)(*[m.ctypes.data for m in ms])
    bv = (ctypes.c_void_p * nd)(*[v.ctypes.data for v in vs])
    apm = [parr(m, ins["idx"], 9) for m in ms]
    bpv = [parr(v, ins["idx"][::-1].copy(), 3) for v in vs]
    apmm = (ctypes.c_void_p * nd)(*[ctypes.cast(x, ctypes.c_void_p).value for x in apm])
    bpvv = (ctypes.c_void_p * nd)(*[ctypes.cast(x, ctypes.c_void_p).value for x in bpv])
    for eq in EQOPS:
        for s1, a_arg in (("nM", am), ("npMa", apmm)):
            for s2, b_arg in (("nV", bv), ("npV", bpvv)):
                name = f"QLA_{pc}_V_v{eq}_{s1}_times_{s2}"
                r = ins["r0V"].copy()
                call(name, ctypes.c_void_p(r.ctypes.data), a_arg, b_arg, N, nd)
                out[name] = r
    # fused spin projection x colour matrix (the Wilson hop terms)
    for mu in range(5):
        for sign in (1, -1):
            for name, dest, bsrc, pb in ((f"QLA_{pc}_D_vpeq_spproj_M_times_pD", "D", "D", True),
                                         (f"QLA_{pc}_H_veq_spproj_Ma_times_D", "H", "D", False),
                                         (f"QLA_{pc}_D_veqm_sprecon_M_times_pH", "D", "H", True),
                                         (f"QLA_{pc}_D_vmeq_spproj_D", "D", "D", False)):
                r = ins["r0" + dest].copy()
                nc_b = 12 if bsrc == "D" else 6
                b = parr(ins[bsrc], ins["idx"], nc_b) if pb else ctypes.c_void_p(ins[bsrc].ctypes.data)
                if name.endswith("_spproj_D"):
                    call(name, ctypes.c_void_p(r.ctypes.data), b, mu, sign, N)
                else:
                    call(name, ctypes.c_void_p(r.ctypes.data), ctypes.c_void_p(ins["M"].ctypes.data), b, mu, sign, N)
                out[f"{name}|{mu}|{sign}"] = r
    # real constant times field
    sc = (ctypes.c_float if dt == np.float32 else ctypes.c_double)(float(ins["scal"][0]))
    for dest, nc in (("V", 3), ("D", 12), ("M", 9)):
        for eq in EQOPS:
            r = ins["r0" + dest].copy()
            call(f"QLA_{pc}_{dest}_v{eq}_r_times_{dest}", ctypes.c_void_p(r.ctypes.data), ctypes.byref(sc),
                 ctypes.c_void_p(ins[dest if dest != "M" else "M2"].ctypes.data), N)
            out[f"QLA_{pc}_{dest}_v{eq}_r_times_{dest}"] = r
    # reductions
    rpcs = [(pc, dt)] + ([("DF3", np.float64)] if pc == "F3" else [])
    for rpc, odt in rpcs:
        for t, nc in (("V", 3), ("H", 6), ("D", 12), ("M", 9)):
            src = ins[t]
            o = np.zeros(1, dtype=odt)
            call(f"QLA_{rpc}_r_veq_norm2_{t}", ctypes.c_void_p(o.ctypes.data), ctypes.c_void_p(src.ctypes.data), N)
            out[f"QLA_{rpc}_r_veq_norm2_{t}"] = o
            o = np.zeros(1, dtype=odt)
            call(f"QLA_{rpc}_r_xeq_norm2_p{t}", ctypes.c_void_p(o.ctypes.data), parr(src, ins["idx"], nc),
                 ctypes.c_void_p(ins["gang"].ctypes.data), N)
            out[f"QLA_{rpc}_r_xeq_norm2_p{t}"] = o
            o = np.zeros(2, dtype=odt)
            b = ins["D2"] if t == "D" else ins["M2"] if t == "M" else ins["r0" + t]
            call(f"QLA_{rpc}_c_veq_{t}_dot_{t}", ctypes.c_void_p(o.ctypes.data), ctypes.c_void_p(src.ctypes.data),
                 ctypes.c_void_p(b.ctypes.data), N)
            out[f"QLA_{rpc}_c_veq_{t}_dot_{t}"] = o
            if rpc != "DF3":
                o = np.zeros(1, dtype=odt)
                call(f"QLA_{rpc}_r_veq_re_{t}_dot_{t}", ctypes.c_void_p(o.ctypes.data),
                     ctypes.c_void_p(src.ctypes.data), ctypes.c_void_p(b.ctypes.data), N)
                out[f"QLA_{rpc}_r_veq_re_{t}_dot_{t}"] = o
    # colour-matrix functions (code templates): exp of anti-Hermitian and of
    # general matrices, sqrt of positive Hermitian, inverse and det of general
    ins["mf_exp"] = T.antihermitian_exp_inputs(rng, N, dt)[0]
    ins["mf_gen"] = (T.gaussian_field(rng, N, 9, dt) * 0.8).astype(dt)
    ins["mf_pos"] = T.positive_hermitian_inputs(rng, N, dt)
    for fname, src in (("M_veq_exp_M", "mf_exp"), ("M_veq_exp_M", "mf_gen"), ("M_veq_sqrt_M", "mf_pos"),
                       ("M_veq_inverse_M", "mf_gen"), ("C_veq_det_M", "mf_gen")):
        r = np.zeros((N, 2 if fname.startswith("C") else 18), dtype=dt)
        call(f"QLA_{pc}_{fname}", ctypes.c_void_p(r.ctypes.data), ctypes.c_void_p(ins[src].ctypes.data), N)
        out[f"QLA_{pc}_{fname}|{src}"] = r
    # the same templates in the N-colour build (FN / DN) at nc = 4 and 8
    npc = "FN" if pc == "F3" else "DN"
    for nc in (4, 8):
        g = (rng.standard_normal((N, 2 * nc * nc)) * (0.25 if nc == 8 else 0.4)).astype(dt)
        pos = T.positive_hermitian_inputs(rng, N, dt, nc=nc)
        ins[f"mfN{nc}_gen"] = g
        ins[f"mfN{nc}_pos"] = pos
        for fname, src in (("M_veq_exp_M", "gen"), ("M_veq_sqrt_M", "pos"), ("M_veq_inverse_M", "gen"),
                           ("C_veq_det_M", "gen")):
            r = np.zeros((N, 2 if fname.startswith("C") else 2 * nc * nc), dtype=dt)
            call(f"QLA_{npc}_{fname}", nc, ctypes.c_void_p(r.ctypes.data),
                 ctypes.c_void_p(ins[f"mfN{nc}_{src}"].ctypes.data), N)
            out[f"QLA_{npc}_{fname}|mfN{nc}_{src}"] = r
    if pc == "F3":
        # the N-colour level-1 loops at nc = 4 and 8 (QLA_FN_ / QLA_DFN_)
        for nc in (4, 8):
            m1 = rng.standard_normal((NS, 2 * nc * nc)).astype(dt)
            vv = rng.standard_normal((NS, 2 * nc)).astype(dt)
            hh = rng.standard_normal((NS, 4 * nc)).astype(dt)
            dd = rng.standard_normal((NS, 8 * nc)).astype(dt)
            r0 = rng.standard_normal((N, 8 * nc)).astype(dt)
            ins.update({f"fn{nc}_M": m1, f"fn{nc}_V": vv, f"fn{nc}_H": hh, f"fn{nc}_D": dd, f"fn{nc}_r0": r0})
            for eq in EQOPS:
                r = r0[:, :2 * nc].copy()
                call(f"QLA_FN_V_v{eq}_M_times_V", nc, ctypes.c_void_p(r.ctypes.data),
                     ctypes.c_void_p(m1.ctypes.data), ctypes.c_void_p(vv.ctypes.data), N)
                out[f"QLA_FN_V_v{eq}_M_times_V|{nc}"] = r
                r = np.ascontiguousarray(np.tile(r0[:, :2 * nc], (1, nc)))
                call(f"QLA_FN_M_v{eq}_Ma_times_pM", nc, ctypes.c_void_p(r.ctypes.data),
                     ctypes.c_void_p(m1.ctypes.data), parr(m1, ins["idx"], nc * nc), N)
                out[f"QLA_FN_M_v{eq}_Ma_times_pM|{nc}"] = r
                for mu in range(5):
                    r = r0[:, :4 * nc].copy()
                    call(f"QLA_FN_H_v{eq}_spproj_D", nc, ctypes.c_void_p(r.ctypes.data),
                         ctypes.c_void_p(dd.ctypes.data), mu, -1, N)
                    out[f"QLA_FN_H_v{eq}_spproj_D|{nc}|{mu}"] = r
                    r = r0[:, :8 * nc].copy()
                    call(f"QLA_FN_D_v{eq}_sprecon_H", nc, ctypes.c_void_p(r.ctypes.data),
                         ctypes.c_void_p(hh.ctypes.data), mu, 1, N)
                    out[f"QLA_FN_D_v{eq}_sprecon_H|{nc}|{mu}"] = r
            vrev = vv[::-1].copy()
            ins[f"fn{nc}_Vrev"] = vrev
            for rpc, odt in (("FN", np.float32), ("DFN", np.float64)):
                o = np.zeros(1, dtype=odt)
                call(f"QLA_{rpc}_r_veq_norm2_D", nc, ctypes.c_void_p(o.ctypes.data), ctypes.c_void_p(dd.ctypes.data), N)
                out[f"QLA_{rpc}_r_veq_norm2_D|{nc}"] = o
                o = np.zeros(2, dtype=odt)
                call(f"QLA_{rpc}_c_veq_V_dot_V", nc, ctypes.c_void_p(o.ctypes.data), ctypes.c_void_p(vv.ctypes.data),
                     ctypes.c_void_p(vrev.ctypes.data), N)
                out[f"QLA_{rpc}_c_veq_V_dot_V|{nc}"] = o
    # the remaining matrix functions (code templates) and a^-1 b
    ins["mf_aht"] = T.from_complex(T.to_complex(ins["mf_exp"].astype(np.float64))
                                   + 1j * rng.uniform(-2, 2, N)[:, None, None] * np.eye(3), dt)
    ins["mf_herm"] = T.hermitian_inputs(rng, N, dt)
    for fname, src in (("M_veq_invsqrt_M", "mf_pos"), ("M_veq_log_M", "mf_pos"), ("M_veq_log_M", "mf_gen"),
                       ("M_veq_expTA_M", "mf_exp"), ("M_veq_expA_M", "mf_aht"), ("M_veq_sqrtPH_M", "mf_pos"),
                       ("M_veq_invsqrtPH_M", "mf_pos"), ("V_veq_eigenvalsH_M", "mf_herm"),
                       ("V_veq_eigenvals_M", "mf_gen")):
        r = np.zeros((N, 6 if fname.startswith("V") else 18), dtype=dt)
        call(f"QLA_{pc}_{fname}", ctypes.c_void_p(r.ctypes.data), ctypes.c_void_p(ins[src].ctypes.data), N)
        out[f"QLA_{pc}_{fname}|{src}"] = r
    for dest in ("V", "M"):
        r = np.zeros((N, 6 if dest == "V" else 18), dtype=dt)
        call(f"QLA_{pc}_{dest}_veq_M_inverse_{dest}", ctypes.c_void_p(r.ctypes.data),
             ctypes.c_void_p(ins["mf_gen"].ctypes.data), ctypes.c_void_p(ins["r0" + dest].ctypes.data), N)
        out[f"QLA_{pc}_{dest}_veq_M_inverse_{dest}|mf_gen|r0{dest}"] = r
    # the N-colour build's generic paths at nc = 4, 8: Newton invsqrt, log and
    # the Hessenberg + QR eigenvalues
    for nc in (4, 8):
        ins[f"mfN{nc}_herm"] = T.hermitian_inputs(rng, N, dt, nc=nc)
        for fname, src in (("M_veq_invsqrt_M", "pos"), ("M_veq_log_M", "pos"), ("V_veq_eigenvals_M", "gen"),
                           ("V_veq_eigenvalsH_M", "herm")):
            r = np.zeros((N, 2 * nc * (1 if fname.startswith("V") else nc)), dtype=dt)
            call(f"QLA_{npc}_{fname}", nc, ctypes.c_void_p(r.ctypes.data),
                 ctypes.c_void_p(ins[f"mfN{nc}_{src}"].ctypes.data), N)
            out[f"QLA_{npc}_{fname}|mfN{nc}_{src}"] = r
    return ins, out


def build_int(seed):
    """Every QLA_I_ v/x entry point of the reference on int_inputs()."""
    import re
    rng = np.random.default_rng(seed)
    R = T.ref()
    ins = T.int_inputs(rng, N, NS)
    names = sorted(set(re.findall(r"void (QLA_I_[vx]\w+) \(", open(os.path.join(
        os.path.dirname(T.REF_SO), "gen", "include", "qla_int.h")).read())))
    out = {}
    keep = []

    def arr(a):
        keep.append(a)
        return ctypes.c_void_p(a.ctypes.data)

    def ptrs(a, idx):
        p = (ctypes.c_void_p * len(idx))(*[a.ctypes.data + 4 * int(j) for j in idx])
        keep.append(p)
        return p

    for name in names:
        r = ins["r0"].copy()
        getattr(R, name)(*T.int_call_args(name, ins, N, arr(r), arr, ptrs))
        out[name] = r
    return ins, out


def main():
    if os.environ.get("OMP_NUM_THREADS") != "1":
        sys.exit("run with OMP_NUM_THREADS=1 (serial reference summation order)")
    if not T.ref_available():
        sys.exit("oracle/_ref/libqla_ref.so missing: run sh oracle/build_ref.sh")
    for pc, dt, seed in (("F3", np.float32, 101), ("D3", np.float64, 202)):
        ins, out = build(pc, dt, seed)
        blob = {"in__" + k: v for k, v in ins.items()}
        blob.update({"out__" + k: v for k, v in out.items()})
        path = os.path.join(HERE, f"qla_{pc.lower()}_golden.npz")
        np.savez_compressed(path, **blob)
        print(f"{path}: {len(out)} reference outputs")
    ins, out = build_int(303)
    blob = {"in__" + k: v for k, v in ins.items()}
    blob.update({"out__" + k: v for k, v in out.items()})
    path = os.path.join(HERE, "qla_int_golden.npz")
    np.savez_compressed(path, **blob)
    print(f"{path}: {len(out)} reference outputs")


if __name__ == "__main__":
    main()
