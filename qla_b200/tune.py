"""Autotuner of the bulk-copy pipeline's launch shape.

    python -m qla_b200.tune [--out qla_b200/tune_b200.txt] [--reps 20] [--keys KEY ...]

For each hot kernel (identified by the key the launcher uses:
"<pc>_<family>:<operand modes>[r]", modes c = contiguous, p = pointer array,
i = int32 index stream, r = destination read by peq/meq) it times every
(consumer threads = sites per tile in {64,128,256}) x (pipeline stages in
{2,3,4}) shape with CUDA events on fields larger than L2 and writes the
fastest per key; the batched program launch (key F3_batch_program, config 4's
64 uneven fields) over sites per tile in {64,128} x stages {2,3,4}.  libqla_b200.so reads the table at its first launch (the
file beside the package, or $QLA_B200_TUNE); keys missing from it use the
built-in heuristic.
"""
import argparse
import ctypes
import itertools
import os
import sys

import qla_b200 as qla

SHAPES = list(itertools.product([64, 128, 256], [2, 3, 4]))
DEFAULT_OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tune_b200.txt")


def _workloads(torch, L):
    """(key, bytes moved per call, callable) for the hot kernels at the sizes
    of the benchmark configurations."""
    V = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    out = []
    for pc, dt, e in (("F3", torch.float32, 1), ("D3", torch.float64, 2)):
        rp = "DF3" if pc == "F3" else "D3"
        n = 48 * 48 * 48 * 96
        x = torch.randn(n, 24, device="cuda", dtype=dt)
        p = torch.randn(n, 24, device="cuda", dtype=dt)
        red = torch.zeros(4, dtype=torch.float64, device="cuda")
        a = (ctypes.c_float if pc == "F3" else ctypes.c_double)(0.25)
        yield (f"{pc}_rtimes_D:cr", 288 * e * n,
               lambda: getattr(L, f"QLA_{pc}_D_vpeq_r_times_D")(V(x), ctypes.byref(a), V(p), n))
        yield (f"{pc}_norm2_D:c", 96 * e * n, lambda: getattr(L, f"QLA_{rp}_r_veq_norm2_D")(V(red), V(x), n))
        yield (f"{pc}_dot_D:cc", 192 * e * n, lambda: getattr(L, f"QLA_{rp}_c_veq_D_dot_D")(V(red), V(x), V(p), n))
        del x, p
        torch.cuda.empty_cache()
        m = 32 * 32 * 32 * 64
        idx = torch.empty(m, dtype=torch.int32, device="cuda")
        qla.shift_index(idx, [32, 32, 32, 64], 0, 1)
        U = torch.randn(m, 18, device="cuda", dtype=dt)
        U2 = torch.randn(m, 18, device="cuda", dtype=dt)
        Mo = torch.randn(m, 18, device="cuda", dtype=dt)
        D = torch.randn(m, 24, device="cuda", dtype=dt)
        H = torch.randn(m, 12, device="cuda", dtype=dt)
        H2 = torch.randn(m, 12, device="cuda", dtype=dt)
        Vv = torch.randn(m, 6, device="cuda", dtype=dt)
        Vo = torch.randn(m, 6, device="cuda", dtype=dt)
        pH = H.data_ptr() + idx.long() * 48 * e
        pV = Vv.data_ptr() + idx.long() * 24 * e
        pM = U2.data_ptr() + idx.long() * 72 * e
        yield (f"{pc}_spproj:c", 144 * e * m, lambda: getattr(L, f"QLA_{pc}_H_veq_spproj_D")(V(H), V(D), 0, 1, m))
        yield (f"{pc}_lmult_H00:ci", (168 * e + 4) * m,
               lambda: getattr(L, f"QLA_{pc}_H_eq_M_times_xH")(V(H2), V(U), V(H), V(idx), m))
        yield (f"{pc}_lmult_H00:cp", (168 * e + 8) * m,
               lambda: getattr(L, f"QLA_{pc}_H_veq_M_times_pH")(V(H2), V(U), V(pH), m))
        yield (f"{pc}_lmult_V00:ci", (120 * e + 4) * m,
               lambda: getattr(L, f"QLA_{pc}_V_eq_M_times_xV")(V(Vo), V(U), V(Vv), V(idx), m))
        yield (f"{pc}_lmult_V00:cp", (120 * e + 8) * m,
               lambda: getattr(L, f"QLA_{pc}_V_veq_M_times_pV")(V(Vo), V(U), V(pV), m))
        yield (f"{pc}_lmult_V00:cc", 120 * e * m,
               lambda: getattr(L, f"QLA_{pc}_V_veq_M_times_V")(V(Vo), V(U), V(Vv), m))
        yield (f"{pc}_lmult_V10:cc", 120 * e * m,
               lambda: getattr(L, f"QLA_{pc}_V_veq_Ma_times_V")(V(Vo), V(U), V(Vv), m))
        yield (f"{pc}_norm2_V:c", 24 * e * m, lambda: getattr(L, f"QLA_{rp}_r_veq_norm2_V")(V(red), V(Vv), m))
        yield (f"{pc}_sprecon:cr", 240 * e * m,
               lambda: getattr(L, f"QLA_{pc}_D_vpeq_sprecon_H")(V(D), V(H2), 0, 1, m))
        Dout = torch.randn(m, 24, device="cuda", dtype=dt)
        yield (f"{pc}_hop_Dspprojfalse:cir", (364 * e - 4 * (e - 1)) * m,
               lambda: getattr(L, f"QLA_{pc}_D_peq_spproj_M_times_xD")(V(Dout), V(U), V(D), V(idx), 0, 1, m))
        yield (f"{pc}_lmult_M00:cp", (216 * e + 8) * m,
               lambda: getattr(L, f"QLA_{pc}_M_veq_M_times_pM")(V(Mo), V(U), V(pM), m))
        yield (f"{pc}_lmult_M00:cc", 216 * e * m,
               lambda: getattr(L, f"QLA_{pc}_M_veq_M_times_M")(V(Mo), V(U), V(U2), m))
        del U, U2, Mo, D, H, H2, Vv, Vo, pH, pV, pM, idx, Dout
        torch.cuda.empty_cache()
    yield _batch_workload(torch)


class _Batch:
    """Config 4's batched launch: 64 F3 fields with extents drawn from
    {8,12,16,20,24,32}^4, each running r = u * u2[nbr], w = r * v.  The tile
    shape is fixed when a plan is built, so prepare() rebuilds the plan after
    each tuned shape is set."""
    SHAPES = list(itertools.product([64, 128], [2, 3, 4]))  # the batch kernel's launch bounds allow 64 / 128

    def __init__(self, torch):
        import numpy as np
        rng = np.random.default_rng(4)
        choices = [8, 12, 16, 20, 24, 32]
        self.fields = []
        for k in range(64):
            dims = [int(x) for x in rng.choice(choices, 4)]
            n = int(np.prod(dims))
            nbr = torch.empty(n, dtype=torch.int32, device="cuda")
            qla.shift_index(nbr, dims, k % 4, 1)
            self.fields.append({"r": torch.empty(n, 18, device="cuda"), "u": torch.randn(n, 18, device="cuda"),
                                "u2": torch.randn(n, 18, device="cuda"), "nbr": nbr,
                                "w": torch.empty(n, 6, device="cuda"), "v": torch.randn(n, 6, device="cuda"),
                                "n": n})
        self.nbytes = sum(f["n"] for f in self.fields) * (72 * 3 + 24 * 2 + 4)
        self.plan = None

    def prepare(self):
        if self.plan is not None:
            self.plan.close()
        self.plan = qla.BatchPlan(self.fields)

    def __call__(self):
        self.plan.run()


def _batch_workload(torch):
    b = _Batch(torch)
    return ("F3_batch_program", b.nbytes, b, _Batch.SHAPES, b.prepare)


def _read_table(path):
    rows = {}
    if os.path.exists(path):
        with open(path) as f:
            for line in f:
                parts = line.split("#")[0].split()
                if len(parts) == 3:
                    g = line.split("#")[1].strip() if "#" in line else "0"
                    rows[parts[0]] = (int(parts[1]), int(parts[2]), float(g or 0))
    return rows


def tune(out=DEFAULT_OUT, reps=20, verbose=True, keys=None):
    """Tune every workload (or those whose key contains one of `keys`, the
    other rows of an existing table kept) and write the table."""
    import torch
    L = qla.lib()
    L.qlagpu_tune_clear()
    rows = []
    for wl in _workloads(torch, L):
        key, nbytes, fn = wl[:3]
        shapes = wl[3] if len(wl) > 3 else SHAPES
        prepare = wl[4] if len(wl) > 4 else None
        if keys and not any(k in key for k in keys):
            continue
        best = None
        for t, s in shapes:
            L.qlagpu_tune_set(key.encode(), t, s)
            if prepare is not None:
                prepare()
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                fn()
            e1.record()
            torch.cuda.synchronize()
            qla.check(key)
            gbs = nbytes / (e0.elapsed_time(e1) / reps) / 1e6
            if best is None or gbs > best[0]:
                best = (gbs, t, s)
        rows.append((key, best[1], best[2], best[0]))
        if verbose:
            print(f"{key:24s} threads {best[1]:3d} stages {best[2]}  {best[0]:7.0f} GB/s", file=sys.stderr)
    L.qlagpu_tune_clear()
    if qla.device_error():
        raise qla.QLAError("a kernel reported an error during tuning")
    table = _read_table(out) if keys else {}
    for key, t, s, g in rows:
        table[key] = (t, s, g)
    _write_table(out, table, torch.cuda.get_device_name())
    return rows


def _write_table(path, table, device):
    """Write {key: (threads, stages, GB/s)} in the format the library reads
    (`key threads stages`, `#` comments)."""
    with open(path, "w") as f:
        f.write("# qla_b200 launch shapes measured on %s by python -m qla_b200.tune\n" % device)
        f.write("# key threads stages  (GB/s of algorithmic traffic at the tuning size)\n")
        for key, (t, s, g) in table.items():
            f.write(f"{key} {t} {s}  # {g:.0f}\n")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--keys", nargs="*", default=None,
                    help="tune only the keys containing one of these strings; keep the table's other rows")
    a = ap.parse_args()
    tune(a.out, a.reps, keys=a.keys)
