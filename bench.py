#!/usr/bin/env python3
"""Benchmark: the mixed-precision CG-style level-1 chain on a 48^3x96
DiracFermion field through the QLA C-ABI of libqla_b200.so.

Workload (one "step"): 50 iterations of
    QLA_F3_D_vpeq_r_times_D(x, &a_k, p)     x += a_k p   (a_k ~ U[-1,1], seeded)
    QLA_DF3_r_veq_norm2_D(&nrm_k, x)        |x|^2, FP64 compensated reduction
    QLA_DF3_c_veq_D_dot_D(&dot_k, x, p)     <x, p>, FP64 compensated reduction
on 10,616,832 sites (x, p: 1.02 GB each in F3, resident in HBM; inputs are far
larger than the 126 MB L2, so no flush is needed between iterations).

metric: site-updates/s, one site-update = one lattice site through one chain
iteration (axpy + norm2 + dot), next to the same chain in plain FP64
(QLA_D3_*) on the same GPU.  Algorithmic bytes per site-update: 576 (F3) and
1152 (D3) (288 axpy + 96 norm2 + 192 dot, x2 for D3).

--impl reference runs the reference's own CPU implementation of the chain
(oracle/_ref/libqla_ref.so, the generated QLA C built with OpenMP) on the
host's cores on a bounded sample of the same field.

Launch: python bench.py [--gpus N --steps K --warmup W]; for N>1 under
torchrun each rank runs an independent replica (QLA is single-node data:
nothing to exchange), value = all ranks' site-updates / max rank time.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

DIMS = (48, 48, 48, 96)
NSITES = 48 * 48 * 48 * 96
ITERS = 50
BYTES_F3 = {"axpy": 288, "norm2": 96, "dot": 192}
BYTES_D3 = {k: 2 * v for k, v in BYTES_F3.items()}
METRIC = "site-updates/s & % B200 HBM peak: FP32+FP64-reduce vs plain FP64, same GPU"
UNIT = "site-updates/s"


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(value, world, device=None):
    """Largest per-rank value (the slowest rank's time) across the job."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, sites, iters, steps, ms_max):
    """Site-updates/s of the whole job: every replica processes `sites`
    sites through `iters` iterations per step; the job takes the slowest
    rank's time."""
    return world * sites * iters * steps / (ms_max / 1e3)


# ---------------------------------------------------------------------------
# clock sampling during the timed region
class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = []
        smax = None
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[1]))
                smax = float(s[2])
            except ValueError:
                continue
            for nm, v in zip(names, s[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def cpu_reference_lib():
    """(ctypes lib, kind): the reference build when present, else the oracle port."""
    ref = os.path.join(REPO, "oracle", "_ref", "libqla_ref.so")
    if os.path.exists(ref):
        return ctypes.CDLL(ref), "reference"
    return ctypes.CDLL(os.path.join(REPO, "oracle", "liboracle.so")), "port"


def cpu_chain_rate(x, p, a_vals, budget_s=15.0, max_iters=None):
    """Time the chain on the host cores: returns (site-updates/s, iterations, seconds, kind, threads)."""
    import numpy as np
    lib, kind = cpu_reference_lib()
    n = x.shape[0]
    xp = ctypes.c_void_p(x.ctypes.data)
    pp = ctypes.c_void_p(p.ctypes.data)
    nrm = ctypes.c_double(0.0)
    dot = (ctypes.c_double * 2)()
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    if kind == "reference":
        axpy, n2, dt = lib.QLA_F3_D_vpeq_r_times_D, lib.QLA_DF3_r_veq_norm2_D, lib.QLA_DF3_c_veq_D_dot_D

        def one(a):
            af = ctypes.c_float(a)
            axpy(xp, ctypes.byref(af), pp, n)
            n2(ctypes.byref(nrm), xp, n)
            dt(dot, xp, pp, n)
    else:
        threads = 1
        lib.ora_rtimes_f.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_long, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        lib.ora_norm2_ref_f.restype = ctypes.c_double

        def one(a):
            lib.ora_rtimes_f(xp, a, pp, n, 12, 1, None, None)
            lib.ora_norm2_ref_f(xp, ctypes.c_long(n), 12, None, None)
            lib.ora_dot_ref_f(dot, xp, pp, ctypes.c_long(n), 12, None, None, None)
    one(float(a_vals[0]))  # warm-up (page faults, thread pool)
    t0 = time.perf_counter()
    it = 0
    while True:
        one(float(a_vals[(it + 1) % len(a_vals)]))
        it += 1
        el = time.perf_counter() - t0
        if el >= budget_s or (max_iters and it >= max_iters):
            break
    return n * it / el, it, el, kind, threads


def reduction_errors(x, p, nrm_v, dot_v, chunk=1 << 20):
    """Relative errors of a GPU norm2 / dot against sums of the same data in
    extended precision: products in long double (exact for float inputs),
    each site's 24 terms summed in long double, sites summed with math.fsum."""
    import math

    import numpy as np
    n2, dr, di = [], [], []
    for i in range(0, x.shape[0], chunk):
        xc = x[i:i + chunk].astype(np.longdouble)
        pc = p[i:i + chunk].astype(np.longdouble)
        xr, xi, pr, pi = xc[:, 0::2], xc[:, 1::2], pc[:, 0::2], pc[:, 1::2]
        n2.append((xc * xc).sum(axis=1).astype(np.float64))
        dr.append((xr * pr + xi * pi).sum(axis=1).astype(np.float64))
        di.append((xr * pi - xi * pr).sum(axis=1).astype(np.float64))
    ref_n = math.fsum(np.concatenate(n2))
    ref_d = complex(math.fsum(np.concatenate(dr)), math.fsum(np.concatenate(di)))
    return {"norm2_rel_err": abs(nrm_v - ref_n) / abs(ref_n),
            "dot_rel_err": abs(complex(*dot_v) - ref_d) / abs(ref_d)}


# ---------------------------------------------------------------------------
def run_reference_arm(args):
    import numpy as np
    rank, world, _ = dist_env()
    if rank != 0:
        return
    os.environ.setdefault("OMP_PROC_BIND", "close")
    rng = np.random.default_rng(7)
    n = NSITES
    x = rng.standard_normal((n, 24), dtype=np.float32)
    p = rng.standard_normal((n, 24), dtype=np.float32)
    a_vals = rng.uniform(-1, 1, ITERS).astype(np.float32)
    per_step_iters = 2  # bounded sample per step
    lib, kind = cpu_reference_lib()
    for _ in range(args.warmup):
        cpu_chain_rate(x, p, a_vals, budget_s=0.0, max_iters=1)
    times = []
    its = 0
    for _ in range(args.steps):
        r, it, el, kind, threads = cpu_chain_rate(x, p, a_vals, budget_s=0.0, max_iters=per_step_iters)
        times.append(el)
        its += it
    tot = sum(times)
    value = n * its / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 sites, f64 reductions",
        "data": "synthetic (seeded N(0,1) DiracFermions, a_k ~ U[-1,1])",
        "config": {"workload": "cg_chain_48^3x96", "sites": n, "iterations_per_step": per_step_iters,
                   "ops": ["QLA_F3_D_vpeq_r_times_D", "QLA_DF3_r_veq_norm2_D", "QLA_DF3_c_veq_D_dot_D"]},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{per_step_iters} chain iterations on the full 48^3x96 field per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def run_gpu_arm(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    import qla_b200 as qla

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    qla.set_stream(stream)
    n = args.sites
    iters = args.iters
    g = torch.Generator(device=dev)
    g.manual_seed(1000 + rank)
    a_vals = np.random.default_rng(7).uniform(-1, 1, ITERS).astype(np.float32)[:iters]
    L = qla.lib()
    fns = {}
    for nm in ("QLA_F3_D_vpeq_r_times_D", "QLA_DF3_r_veq_norm2_D", "QLA_DF3_c_veq_D_dot_D",
               "QLA_D3_D_vpeq_r_times_D", "QLA_D3_r_veq_norm2_D", "QLA_D3_c_veq_D_dot_D"):
        fns[nm] = getattr(L, nm)
        fns[nm].restype = None
    chain_f = (fns["QLA_F3_D_vpeq_r_times_D"], fns["QLA_DF3_r_veq_norm2_D"], fns["QLA_DF3_c_veq_D_dot_D"],
               [ctypes.c_float(float(v)) for v in a_vals])
    chain_d = (fns["QLA_D3_D_vpeq_r_times_D"], fns["QLA_D3_r_veq_norm2_D"], fns["QLA_D3_c_veq_D_dot_D"],
               [ctypes.c_double(float(v)) for v in a_vals])
    nrm = torch.zeros(iters, dtype=torch.float64, device=dev)
    dot = torch.zeros(iters, 2, dtype=torch.float64, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def chain(xa, pa, ch, ev=None):
        """One step: `iters` iterations of axpy, norm2, dot; reduction results
        stay on the device (asynchronous calls)."""
        axpy, n2, dt, avals = ch
        xp, pp = ctypes.c_void_p(xa.data_ptr()), ctypes.c_void_p(pa.data_ptr())
        nb, db = nrm.data_ptr(), dot.data_ptr()
        for k in range(iters):
            if ev is not None:
                ev[k][0].record(stream)
            axpy(xp, ctypes.byref(avals[k]), pp, n)
            if ev is not None:
                ev[k][1].record(stream)
            n2(ctypes.c_void_p(nb + 8 * k), xp, n)
            if ev is not None:
                ev[k][2].record(stream)
            dt(ctypes.c_void_p(db + 16 * k), xp, pp, n)
            if ev is not None:
                ev[k][3].record(stream)

    def timed(xa, pa, ch):
        """Device time of K steps after W warm-up steps (CUDA events on the
        launching stream, barrier + synchronize on both sides), plus the
        average duration of each of the three kernels (events around every
        launch inside the timed region)."""
        for _ in range(args.warmup):
            chain(xa, pa, ch)
        qla.check("warm-up")
        evs = []
        barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(args.steps):
            ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(iters)]
            chain(xa, pa, ch, ev)
            evs.append(ev)
        t1.record(stream)
        barrier()
        ms = t0.elapsed_time(t1)
        kern = {"axpy": 0.0, "norm2": 0.0, "dot": 0.0}
        for ev in evs:
            for k in range(iters):
                kern["axpy"] += ev[k][0].elapsed_time(ev[k][1])
                kern["norm2"] += ev[k][1].elapsed_time(ev[k][2])
                kern["dot"] += ev[k][2].elapsed_time(ev[k][3])
        nl = max(1, len(evs) * iters)
        qla.check("timed region")
        if qla.device_error():
            raise qla.QLAError("a kernel reported an error in the timed region")
        return ms, {k: v / nl for k, v in kern.items()}

    # ---------------- FP32 sites + FP64 reductions chain (F3 / DF3)
    x = torch.randn(n, 24, device=dev, dtype=torch.float32, generator=g)
    p = torch.randn(n, 24, device=dev, dtype=torch.float32, generator=g)
    clk = ClockSampler(local)
    clk.start()
    ms_f, kern_f = timed(x, p, chain_f)
    clocks = clk.stop()
    ms_f = max_over_ranks(ms_f, world, dev)
    value = whole_job_rate(world, n, iters, args.steps, ms_f)
    assert np.all(np.isfinite(nrm.cpu().numpy()))
    # accuracy of the last iteration's reductions (x as the last axpy left it)
    red_err = None
    if not args.no_accuracy:
        red_err = reduction_errors(x.cpu().numpy(), p.cpu().numpy(), float(nrm[iters - 1]),
                                   dot[iters - 1].cpu().numpy())

    # ---------------- end to end through the C-ABI with host buffers: per step
    # the pinned host -> device copy of x and p, the chain, and the device ->
    # host read of the 3*iters reduction results.  The inputs are double
    # buffered: step s+1's copy runs on a copy stream while step s computes
    # (it waits until step s-1, the last user of that buffer, has finished);
    # the serial figure (copy, then compute) is reported beside it.
    e2e = None
    if not args.no_e2e:
        xh = torch.empty((n, 24), dtype=torch.float32, pin_memory=True)
        ph = torch.empty((n, 24), dtype=torch.float32, pin_memory=True)
        xh.copy_(x)
        ph.copy_(p)
        nrm_h = torch.empty(iters, dtype=torch.float64, pin_memory=True)
        dot_h = torch.empty((iters, 2), dtype=torch.float64, pin_memory=True)
        # the same K steps as the device-timed value: the first step's upload
        # has nothing to overlap with, and K steps amortise it as the chain's
        # own timing does
        e_steps = max(1, args.steps)
        xs, ps = [x, torch.empty_like(x)], [p, torch.empty_like(p)]
        cstream = torch.cuda.Stream(device=dev)
        ready = [torch.cuda.Event() for _ in range(2)]
        free = [torch.cuda.Event() for _ in range(2)]

        def upload(b, after=None):
            if after is not None:
                cstream.wait_event(after)
            cstream.wait_event(free[b])
            with torch.cuda.stream(cstream):
                xs[b].copy_(xh, non_blocking=True)
                ps[b].copy_(ph, non_blocking=True)
            ready[b].record(cstream)

        def compute(b):
            stream.wait_event(ready[b])
            chain(xs[b], ps[b], chain_f)
            free[b].record(stream)
            nrm_h.copy_(nrm, non_blocking=True)
            dot_h.copy_(dot, non_blocking=True)

        def timed_e2e(overlap):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            barrier()
            e0.record(stream)
            if overlap:
                upload(0, after=e0)
                for s_ in range(e_steps):
                    if s_ + 1 < e_steps:
                        upload((s_ + 1) % 2)
                    compute(s_ % 2)
            else:
                for _ in range(e_steps):
                    mark = torch.cuda.Event()
                    mark.record(stream)
                    upload(0, after=mark)
                    compute(0)
            e1.record(stream)
            barrier()
            return max_over_ranks(e0.elapsed_time(e1), world, dev)

        upload(0)
        compute(0)
        upload(1)
        compute(1)
        ms_serial = timed_e2e(False)
        ms_e = timed_e2e(True)
        qla.check("e2e")
        e2e = {"value": whole_job_rate(world, n, iters, e_steps, ms_e), "unit": UNIT,
               "h2d_bytes_per_step": int(xh.numel() * 4 + ph.numel() * 4),
               "d2h_bytes_per_step": int(nrm_h.numel() * 8 + dot_h.numel() * 8), "steps": e_steps,
               "ms_per_step": ms_e / e_steps, "overlap": "double-buffered inputs, copy stream",
               "serial_value": whole_job_rate(world, n, iters, e_steps, ms_serial)}
        del xh, ph, xs, ps
    del x, p
    torch.cuda.empty_cache()

    # ---------------- plain FP64 chain (D3) on the same GPU
    value_d = ms_d = None
    kern_d = {}
    if not args.no_fp64:
        xd = torch.randn(n, 24, device=dev, dtype=torch.float64, generator=g)
        pd = torch.randn(n, 24, device=dev, dtype=torch.float64, generator=g)
        ms_d, kern_d = timed(xd, pd, chain_d)
        ms_d = max_over_ranks(ms_d, world, dev)
        value_d = whole_job_rate(world, n, iters, args.steps, ms_d)
        if red_err is not None:
            ed = reduction_errors(xd.cpu().numpy(), pd.cpu().numpy(), float(nrm[iters - 1]),
                                  dot[iters - 1].cpu().numpy())
            red_err.update({"fp64_chain_" + k: v for k, v in ed.items()})
        del xd, pd
        torch.cuda.empty_cache()

    # ---------------- roofline: algorithmic bytes per launch / event-timed duration
    peak, peak_kind = peaks()

    # ---------------- the other north-star targets on the same GPU (N=1):
    # config-2 per-kernel HBM fractions and the hop sequence, config-4 batched
    # launch (its HBM fraction and its uneven / equal-volume ratio), the
    # DiracPropagator products and the F3 matrix exp; CUDA events on the
    # launching stream, inputs larger than L2
    extra = {}
    if world == 1 and not args.no_extra:
        reps = max(args.steps, 5)
        extra["config2_hop"] = hop_figures(torch, qla, qla.lib(), stream, peak, reps)
        torch.cuda.empty_cache()
        extra["config4_batched"] = batched_figures(torch, qla, qla.lib(), stream, peak, reps)
        torch.cuda.empty_cache()
        extra["prop_and_exp"] = prop_mfunc_figures(torch, qla, qla.lib(), stream, peak, reps)
        torch.cuda.empty_cache()
        qla.check("secondary configurations")
        if qla.device_error():
            raise qla.QLAError("a kernel reported an error in the secondary configurations")

    def roof(kern, bytes_tab):
        out = {}
        for nm, ms in kern.items():
            ach = bytes_tab[nm] * n / (ms / 1e3) / 1e9
            out[nm] = {"achieved_gbs": ach, "frac": ach / peak, "us_per_launch": 1e3 * ms}
        return out

    rl = roof(kern_f, BYTES_F3)
    rl_d = roof(kern_d, BYTES_D3)
    dom = max(kern_f, key=lambda k: kern_f[k])
    kname = {"axpy": "QLA_F3_D_vpeq_r_times_D", "norm2": "QLA_DF3_r_veq_norm2_D", "dot": "QLA_DF3_c_veq_D_dot_D"}
    traffic = None
    tp = os.path.join(REPO, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get(kname[dom])
    chain_bytes = sum(BYTES_F3.values())

    # ---------------- CPU baseline (rank 0, N=1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        xs = np.random.default_rng(3).standard_normal((n, 24), dtype=np.float32)
        ps = np.random.default_rng(4).standard_normal((n, 24), dtype=np.float32)
        os.environ.setdefault("OMP_PROC_BIND", "close")
        r, it, el, kind, threads = cpu_chain_rate(xs, ps, a_vals, budget_s=args.cpu_seconds)
        cpu = {"value": r, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"{it} chain iterations on the full {n}-site field ({el:.1f} s)"}
        if kind == "reference":
            # the same chain on one host thread (the reference's OpenMP
            # runtime set to one thread for this sample, then restored)
            try:
                gomp = ctypes.CDLL("libgomp.so.1")
                gomp.omp_set_num_threads(1)
                r1, it1, el1, _, _ = cpu_chain_rate(xs, ps, a_vals, budget_s=min(5.0, args.cpu_seconds))
                gomp.omp_set_num_threads(threads)
                cpu["single_thread"] = {"value": r1, "unit": UNIT,
                                        "sample": f"{it1} chain iterations ({el1:.1f} s)"}
            except OSError:
                pass

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_f / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 sites, f64 reductions",
            "data": "synthetic (seeded N(0,1) DiracFermions, a_k ~ U[-1,1])",
            "config": {"workload": "cg_chain_48^3x96" if n == NSITES else f"cg_chain_{n}_sites", "sites": n,
                       "iterations_per_step": iters,
                       "ops": ["QLA_F3_D_vpeq_r_times_D", "QLA_DF3_r_veq_norm2_D", "QLA_DF3_c_veq_D_dot_D"],
                       "bytes_per_site_update": chain_bytes, "l2": "inputs (2 x 1.02 GB) larger than L2, no flush",
                       "parallelism": f"replicas x{world}"},
            "hbm_frac_chain": value / world * chain_bytes / 1e9 / peak,
            "fp64_chain": None if value_d is None else {
                "value": value_d, "ms_per_step": ms_d / args.steps,
                "hbm_frac": value_d / world * 2 * chain_bytes / 1e9 / peak,
                "ops": ["QLA_D3_D_vpeq_r_times_D", "QLA_D3_r_veq_norm2_D", "QLA_D3_c_veq_D_dot_D"],
                "kernels": rl_d},
            "speedup_vs_fp64": None if value_d is None else value / value_d,
            "roofline": {"bound": "hbm", "kernel": kname[dom], "achieved": rl[dom]["achieved_gbs"], "peak": peak,
                         "unit": "GB/s", "frac": rl[dom]["frac"], "peak_kind": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_launch": BYTES_F3[dom] * n},
            "kernels": rl,
            "reductions": None if red_err is None else dict(
                red_err, reference="the same data in long double (exact products for float inputs), "
                                   "sites summed with math.fsum; last iteration of the timed region"),
            "e2e": e2e,
            "gpu_launches": 3 * iters * args.steps,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# secondary workloads (configs 1, 2, 4, 5 of the level-1 study): one JSON line each, same
# timing rules (warm-up, CUDA events on the launching stream, inputs > L2
# unless stated).  The default workload above is the benchmark line.
def _events_time(torch, stream, fn, reps, warmup=3):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def hop_figures(torch, qla, L, stream, peak, reps):
    """Config 2: the Wilson-hop-shaped sequence on the 32^3x64 periodic lattice
    (8 x spproj -> M_times_xH -> vpeq_sprecon), the fused hop term, the
    4-direction nM_times_npV, and each kernel of the sequence timed alone;
    F3 and D3.  Returns the workload's JSON fields."""
    import numpy as np
    V = lambda t: ctypes.c_void_p(t if isinstance(t, int) else t.data_ptr())  # noqa: E731
    out = {}
    dims = [32, 32, 32, 64]
    n = int(np.prod(dims))
    res = {}
    for pc, dt, e in (("F3", torch.float32, 1), ("D3", torch.float64, 2)):
        D = torch.randn(n, 24, device="cuda", dtype=dt)
        Out = torch.zeros(n, 24, device="cuda", dtype=dt)
        H = torch.empty(n, 12, device="cuda", dtype=dt)
        H2 = torch.empty(n, 12, device="cuda", dtype=dt)
        U = [torch.randn(n, 18, device="cuda", dtype=dt) for _ in range(4)]
        Vv = torch.randn(n, 6, device="cuda", dtype=dt)
        Vo = torch.empty(n, 6, device="cuda", dtype=dt)
        nbr = {}
        for mu in range(4):
            for sg in (1, -1):
                nbr[(mu, sg)] = torch.empty(n, dtype=torch.int32, device="cuda")
                qla.shift_index(nbr[(mu, sg)], dims, mu, sg)
        sp, mh, rc = (getattr(L, f"QLA_{pc}_H_veq_spproj_D"), getattr(L, f"QLA_{pc}_H_eq_M_times_xH"),
                      getattr(L, f"QLA_{pc}_D_vpeq_sprecon_H"))

        def hop():
            for mu in range(4):
                for sg in (1, -1):
                    sp(V(H), V(D), mu, sg, n)
                    mh(V(H2), V(U[mu]), V(H), V(nbr[(mu, sg)]), n)
                    rc(V(Out), V(H2), mu, sg, n)
        ms = _events_time(torch, stream, hop, reps)
        fz = getattr(L, f"QLA_{pc}_D_peq_spproj_M_times_xD")

        def hop_fused():
            for mu in range(4):
                for sg in (1, -1):
                    fz(V(Out), V(U[mu]), V(D), V(nbr[(mu, sg)]), mu, sg, n)
        ms_f = _events_time(torch, stream, hop_fused, reps)
        # staggered-style 4-direction sum r += sum_mu U_mu V[x+mu] through
        # QLA's pointer form (QLA_<pc>_V_vpeq_nM_times_npV, nd = 4)
        pv = [(Vv.data_ptr() + nbr[(mu, 1)].long() * 24 * e).contiguous() for mu in range(4)]
        tab_a = (ctypes.c_void_p * 4)(*[U[mu].data_ptr() for mu in range(4)])
        tab_b = (ctypes.c_void_p * 4)(*[t.data_ptr() for t in pv])
        nmv = getattr(L, f"QLA_{pc}_V_vpeq_nM_times_npV")
        ms_nm = _events_time(torch, stream, lambda: nmv(V(Vo), tab_a, tab_b, n, 4), reps * 4)
        t_sp = _events_time(torch, stream, lambda: sp(V(H), V(D), 0, 1, n), reps * 4)
        t_mh = _events_time(torch, stream, lambda: mh(V(H2), V(U[0]), V(H), V(nbr[(0, 1)]), n), reps * 4)
        t_rc = _events_time(torch, stream, lambda: rc(V(Out), V(H2), 0, 1, n), reps * 4)
        mv = getattr(L, f"QLA_{pc}_V_eq_M_times_xV")
        t_mv = _events_time(torch, stream, lambda: mv(V(Vo), V(U[0]), V(Vv), V(nbr[(0, 1)]), n), reps * 4)
        ptrs = (Vv.data_ptr() + nbr[(0, 1)].long() * 24 * e).contiguous()
        mvp = getattr(L, f"QLA_{pc}_V_veq_M_times_pV")
        t_mvp = _events_time(torch, stream, lambda: mvp(V(Vo), V(U[0]), V(ptrs), n), reps * 4)
        qla.check("hop")
        b = {"spproj": 144 * e, "M_times_xH": 168 * e + 4, "sprecon": 240 * e, "M_times_xV": 120 * e + 4,
             "M_times_pV": 120 * e + 8}
        tk = {"spproj": t_sp, "M_times_xH": t_mh, "sprecon": t_rc, "M_times_xV": t_mv, "M_times_pV": t_mvp}
        res[pc] = {"site_updates_per_s": n / (ms / 1e3), "ms_per_hop": ms,
                   "nM_times_npV_nd4": {"us": 1e3 * ms_nm, "gbs": (4 * (72 * e + 8 + 24 * e) + 48 * e) * n /
                                        (ms_nm / 1e3) / 1e9,
                                        "frac": (4 * (72 * e + 8 + 24 * e) + 48 * e) * n / (ms_nm / 1e3) / 1e9
                                        / peak},
                   "fused": {"op": f"QLA_{pc}_D_peq_spproj_M_times_xD", "ms_per_hop": ms_f,
                             "site_updates_per_s": n / (ms_f / 1e3),
                             "hbm_frac": n * 8 * (364 * e) / (ms_f / 1e3) / 1e9 / peak,
                             "speedup_vs_unfused": ms / ms_f},
                   "hbm_frac_hop": n * 8 * sum(b[k] for k in ("spproj", "M_times_xH", "sprecon")) / (ms / 1e3)
                   / 1e9 / peak,
                   "kernels": {k: {"us": 1e3 * tk[k], "gbs": b[k] * n / (tk[k] / 1e3) / 1e9,
                                   "frac": b[k] * n / (tk[k] / 1e3) / 1e9 / peak} for k in tk}}
        del D, Out, H, H2, U, Vv, Vo, nbr, ptrs, pv
        torch.cuda.empty_cache()
    out.update({"metric": "Wilson-hop level-1 sequence (8 x spproj, M_times_xH, vpeq_sprecon), 32^3x64",
                "unit": "site-updates/s", "value": res["F3"]["site_updates_per_s"], "F3": res["F3"],
                "D3": res["D3"], "speedup_vs_fp64": res["F3"]["ms_per_hop"] and
                res["D3"]["ms_per_hop"] / res["F3"]["ms_per_hop"]})
    return out


def batched_figures(torch, qla, L, stream, peak, reps):
    """Config 4: 64 F3 fields of uneven extents in one persistent launch
    replayed from a CUDA graph, against 128 separate launches and an
    equal-volume batch of the same total.  Returns the workload's JSON fields."""
    import numpy as np
    V = lambda t: ctypes.c_void_p(t if isinstance(t, int) else t.data_ptr())  # noqa: E731
    out = {}
    rng = np.random.default_rng(4)
    choices = [8, 12, 16, 20, 24, 32]
    dims_list = [[int(x) for x in rng.choice(choices, 4)] for _ in range(64)]
    vols = [int(np.prod(d)) for d in dims_list]

    def make(dlist):
        """one field per lattice: links u, u2, vector v, +mu neighbour table"""
        fl = []
        for k, dims in enumerate(dlist):
            n = int(np.prod(dims))
            nbr = torch.empty(n, dtype=torch.int32, device="cuda")
            qla.shift_index(nbr, dims, k % 4, 1)
            fl.append({"r": torch.empty(n, 18, device="cuda"), "u": torch.randn(n, 18, device="cuda"),
                       "u2": torch.randn(n, 18, device="cuda"), "nbr": nbr,
                       "w": torch.empty(n, 6, device="cuda"), "v": torch.randn(n, 6, device="cuda"), "n": n})
        return fl
    tot = sum(vols)
    uneven = make(dims_list)
    plan = qla.BatchPlan(uneven)
    g = torch.cuda.CUDAGraph()
    s2 = torch.cuda.Stream()
    with torch.cuda.stream(s2):
        qla.set_stream(s2)
        plan.run()
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=s2):
            plan.run()
    qla.set_stream(stream)
    ms_b = _events_time(torch, stream, g.replay, reps)
    mxm, mxv = L.QLA_F3_M_eq_M_times_xM, L.QLA_F3_V_veq_M_times_V

    def separate():
        for f in uneven:
            mxm(V(f["r"]), V(f["u"]), V(f["u2"]), V(f["nbr"]), f["n"])
            mxv(V(f["w"]), V(f["r"]), V(f["v"]), f["n"])
    ms_s = _events_time(torch, stream, separate, reps)
    del g
    plan.close()
    del uneven
    torch.cuda.empty_cache()
    # equal-volume batch of the same total: 64 lattices 16x16x16xLt
    lt = max(1, round(tot / 64 / 4096))
    even_n = 4096 * lt
    even = make([[16, 16, 16, lt]] * 64)
    plan_e = qla.BatchPlan(even)
    ms_e = _events_time(torch, stream, plan_e.run, reps)
    plan_e.close()
    qla.check("batched")
    rate_b = tot / (ms_b / 1e3)
    rate_e = 64 * even_n / (ms_e / 1e3)
    out.update({"metric": "batched uneven-volume M_times_xM + M_times_V (64 F3 fields, extents in "
                          "{8..32}^4), one persistent launch replayed from a CUDA graph",
                "unit": "site-updates/s", "value": rate_b, "total_sites": tot,
                "ms_batched_graph": ms_b, "ms_128_separate_launches": ms_s,
                "speedup_vs_separate": ms_s / ms_b, "equal_volume_rate": rate_e,
                "uneven_vs_equal_volume": rate_b / rate_e,
                "hbm_frac": rate_b * (72 * 3 + 24 * 2 + 4) / 1e9 / peak,
                "bytes_per_site": "U 72 + U2 gather 72 + nbr 4 + V 24 + R 72 + W 24 = 268"})
    return out


def prop_mfunc_figures(torch, qla, L, stream, peak, reps):
    """The DiracPropagator products P*P and P^+*P (16^3x32 sites, 3456
    algorithmic bytes per site F3) and the F3 matrix exp (32^3x64 sites of
    i Q, Q traceless Hermitian with Frobenius norm uniform in [0, 3 sqrt 2];
    144 bytes per site), CUDA events on the launching stream, inputs larger
    than L2."""
    V = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    out = {}
    n = 16 * 16 * 16 * 32
    for pc, dt, e in (("F3", torch.float32, 4), ("D3", torch.float64, 8)):
        pa = torch.randn(n, 288, device="cuda", dtype=dt)
        pb = torch.randn(n, 288, device="cuda", dtype=dt)
        pr = torch.empty(n, 288, device="cuda", dtype=dt)
        for nm in ("P_veq_P_times_P", "P_veq_Pa_times_P"):
            f = getattr(L, f"QLA_{pc}_{nm}")
            ms = _events_time(torch, stream, lambda f=f: f(V(pr), V(pa), V(pb), n), reps)
            gbs = 3 * 288 * e * n / (ms / 1e3) / 1e9
            out[f"{pc}_{nm}"] = {"site_updates_per_s": n / (ms / 1e3), "us": 1e3 * ms, "gbs": gbs,
                                 "hbm_frac": gbs / peak, "sites": n}
        del pa, pb, pr
    n = 32 * 32 * 32 * 64
    q = torch.randn(n, 3, 3, device="cuda", dtype=torch.complex128)
    q = 0.5 * (q + q.conj().transpose(1, 2))
    q = q - (torch.diagonal(q, dim1=1, dim2=2).sum(-1) / 3)[:, None, None] * torch.eye(3, device="cuda")
    fro = torch.sqrt((q.abs() ** 2).sum(dim=(1, 2)))
    q = q * (torch.rand(n, device="cuda", dtype=torch.float64) * 3 * 2 ** 0.5 / fro)[:, None, None]
    a = torch.view_as_real((1j * q).reshape(n, 9)).reshape(n, 18).to(torch.float32).contiguous()
    r = torch.empty_like(a)
    del q
    ms = _events_time(torch, stream, lambda: L.QLA_F3_M_veq_exp_M(V(r), V(a), n), reps)
    out["F3_M_veq_exp_M"] = {"site_updates_per_s": n / (ms / 1e3), "us": 1e3 * ms,
                             "gbs": 144 * n / (ms / 1e3) / 1e9, "sites": n,
                             "note": "FP64 Cayley-Hamilton coefficients, FP32 assembly and squarings"}
    del a, r
    return out


def run_workload(args):
    import numpy as np
    import torch

    import qla_b200 as qla
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    qla.set_stream(stream)
    peak, peak_kind = peaks()
    L = qla.lib()
    V = lambda t: ctypes.c_void_p(t if isinstance(t, int) else t.data_ptr())  # noqa: E731
    out = {"workload": args.workload, "peak_gbs": peak, "peak_kind": peak_kind, "data": "synthetic, seeded"}
    reps = max(args.steps, 5)
    if args.workload == "hop":
        out.update(hop_figures(torch, qla, L, stream, peak, reps))
    elif args.workload == "batched":
        out.update(batched_figures(torch, qla, L, stream, peak, reps))
    elif args.workload == "mfunc":
        # every colour-matrix function of the code templates on 32^3x64
        # sites; the reference library (host cores, OpenMP) on a 32,768-site
        # sample of the same inputs beside it
        n = 32 * 32 * 32 * 64
        ns = 32768
        res = {}
        lib_cpu, cpu_kind = cpu_reference_lib()
        threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
        eye = torch.eye(3, device="cuda", dtype=torch.complex128)

        def as_field(z, dt):
            return torch.view_as_real(z.reshape(n, 9)).reshape(n, 18).to(dt).contiguous()

        for pc, dt in (("F3", torch.float32), ("D3", torch.float64)):
            g = torch.randn(n, 3, 3, device="cuda", dtype=torch.complex128) * 0.5
            gh = g.conj().transpose(1, 2)
            ins = {"gen": as_field(g, dt), "pos": as_field(gh @ g + 0.1 * eye, dt),
                   "ah": as_field(0.5 * (g - gh), dt), "herm": as_field(0.5 * (g + gh), dt)}
            tl = 0.5 * (g - gh)
            tl = tl - (torch.diagonal(tl, dim1=1, dim2=2).sum(-1) / 3)[:, None, None] * eye
            ins["ahtl"] = as_field(tl, dt)
            del g, gh, tl
            bv = torch.randn(n, 6, device="cuda", dtype=dt)
            e = 4 if pc == "F3" else 8
            rM = torch.empty(n, 18, device="cuda", dtype=dt)
            rV = torch.empty(n, 6, device="cuda", dtype=dt)
            rC = torch.empty(n, 2, device="cuda", dtype=dt)
            table = [("exp", "M", "ahtl", rM, 36), ("expTA", "M", "ahtl", rM, 36), ("expA", "M", "ah", rM, 36),
                     ("sqrt", "M", "pos", rM, 36), ("invsqrt", "M", "pos", rM, 36), ("sqrtPH", "M", "pos", rM, 36),
                     ("invsqrtPH", "M", "pos", rM, 36), ("log", "M", "pos", rM, 36), ("inverse", "M", "gen", rM, 36),
                     ("det", "C", "gen", rC, 20), ("eigenvalsH", "V", "herm", rV, 24),
                     ("eigenvals", "V", "gen", rV, 24), ("M_inverse_V", "V", "gen", rV, 30),
                     ("M_inverse_M", "M", "gen", rM, 54)]
            for fname, dest, src, outt, nb in table:
                if fname.startswith("M_inverse"):
                    bb = bv if dest == "V" else ins["pos"]
                    f = getattr(L, f"QLA_{pc}_{dest}_veq_{fname}")
                    call = (lambda f=f, outt=outt, src=src, bb=bb: f(V(outt), V(ins[src]), V(bb), n))
                else:
                    f = getattr(L, f"QLA_{pc}_{dest}_veq_{fname}_M")
                    call = (lambda f=f, outt=outt, src=src: f(V(outt), V(ins[src]), n))
                ms = _events_time(torch, stream, call, reps)
                row = {"site_updates_per_s": n / (ms / 1e3), "us": 1e3 * ms, "gbs": nb * e * n / (ms / 1e3) / 1e9}
                if cpu_kind == "reference":
                    a_h = ins[src][:ns].cpu().numpy()
                    o_h = np.zeros((ns, outt.shape[1]), dtype=a_h.dtype)
                    fc = getattr(lib_cpu, f.__name__)
                    if fname.startswith("M_inverse"):
                        b_h = bb[:ns].cpu().numpy()
                        cc = (lambda fc=fc: fc(V(o_h.ctypes.data), V(a_h.ctypes.data), V(b_h.ctypes.data), ns))
                    else:
                        cc = (lambda fc=fc: fc(V(o_h.ctypes.data), V(a_h.ctypes.data), ns))
                    cc()
                    t0 = time.perf_counter()
                    it = 0
                    while time.perf_counter() - t0 < 0.4:
                        cc()
                        it += 1
                    cpu = ns * it / (time.perf_counter() - t0)
                    row["cpu_site_updates_per_s"] = cpu
                    row["gpu_over_cpu"] = row["site_updates_per_s"] / cpu
                res[f"{pc}_{fname}"] = row
            qla.check("mfunc")
            del ins, bv, rM, rV, rC
            torch.cuda.empty_cache()
        out.update({"metric": "colour-matrix functions on 32^3x64 sites (every function of the code templates)",
                    "unit": "site-updates/s", "value": res["F3_exp"]["site_updates_per_s"], "ops": res,
                    "cpu_baseline": {"kind": cpu_kind, "cores": threads,
                                     "sample": f"{ns} sites of the same inputs, repeated for 0.4 s per op"}})
    elif args.workload == "prop":
        # DiracPropagator products (1152-B F3 records): M*P, P*M, P*P, P^+*P
        # (peq forms read the destination too) and the spin trace, 16^3x32
        n = 16 * 16 * 16 * 32
        res = {}
        for pc, dt, e in (("F3", torch.float32, 4), ("D3", torch.float64, 8)):
            m = torch.randn(n, 18, device="cuda", dtype=dt)
            pa = torch.randn(n, 288, device="cuda", dtype=dt)
            pb = torch.randn(n, 288, device="cuda", dtype=dt)
            pr = torch.randn(n, 288, device="cuda", dtype=dt)
            mr = torch.empty(n, 18, device="cuda", dtype=dt)
            P = 288 * e  # bytes of one propagator record
            table = [("P_veq_M_times_P", (pr, m, pa), 9 * 2 * e + 2 * P),
                     ("P_veq_P_times_M", (pr, pa, m), 9 * 2 * e + 2 * P),
                     ("P_vpeq_M_times_P", (pr, m, pa), 9 * 2 * e + 3 * P),
                     ("P_veq_P_times_P", (pr, pa, pb), 3 * P),
                     ("P_veq_Pa_times_P", (pr, pa, pb), 3 * P),
                     ("M_veq_spintrace_P", (mr, pa), P + 9 * 2 * e)]
            for nm, args_, nb in table:
                f = getattr(L, f"QLA_{pc}_{nm}")
                call = (lambda f=f, args_=args_: f(*[V(t) for t in args_], n))
                ms = _events_time(torch, stream, call, reps)
                gbs = nb * n / (ms / 1e3) / 1e9
                res[f"{pc}_{nm}"] = {"site_updates_per_s": n / (ms / 1e3), "us": 1e3 * ms, "bytes_per_site": nb,
                                     "gbs": gbs, "hbm_frac": gbs / peak}
            qla.check("prop")
            del m, pa, pb, pr, mr
            torch.cuda.empty_cache()
        out.update({"metric": "DiracPropagator products and spin trace on 16^3x32 sites", "unit": "site-updates/s",
                    "value": res["F3_P_veq_M_times_P"]["site_updates_per_s"], "ops": res})
    elif args.workload == "ewise":
        # element-wise families and site-local products on 32^3x64 sites
        n = 32 * 32 * 32 * 64
        res = {}
        for pc, dt, e in (("F3", torch.float32, 4), ("D3", torch.float64, 8)):
            D = lambda: torch.randn(n, 24, device="cuda", dtype=dt)  # noqa: E731
            x, y, z = D(), D(), D()
            m1, m2 = torch.randn(n, 18, device="cuda", dtype=dt), torch.randn(n, 18, device="cuda", dtype=dt)
            cf = torch.randn(n, 2, device="cuda", dtype=dt)
            cs = torch.tensor([0.3, -0.7], device="cuda", dtype=dt)
            ps = torch.randn(n // 8, 288, device="cuda", dtype=dt)
            pr = torch.empty_like(ps)
            rr = torch.empty(n // 8, device="cuda", dtype=dt)
            table = [("D_vpeq_c_times_D", (x, cs, y), n, 288),
                     ("D_veq_c_times_D_plus_D", (z, cs, x, y), n, 288),
                     ("D_veq_C_times_D", (z, cf, x), n, 200),
                     ("M_veq_Ca_times_Ma", (m1, cf, m2), n, 152),
                     ("C_vpeq_D_dot_D", (cf, x, y), n, 208),
                     ("P_veq_c_times_P", (pr, cs, ps), n // 8, 2304),
                     ("R_veq_norm2_P", (rr, ps), n // 8, 1156)]
            for nm, targs, nn, nb in table:
                f = getattr(L, f"QLA_{pc}_{nm}")
                call = (lambda f=f, targs=targs, nn=nn: f(*[V(t) for t in targs], nn))
                ms = _events_time(torch, stream, call, reps)
                gbs = nb * (e // 4) * nn / (ms / 1e3) / 1e9
                res[f"{pc}_{nm}"] = {"site_updates_per_s": nn / (ms / 1e3), "us": 1e3 * ms, "gbs": gbs,
                                     "hbm_frac": gbs / peak}
            qla.check("ewise")
            del x, y, z, m1, m2, cf, ps, pr, rr
            torch.cuda.empty_cache()
        out.update({"metric": "element-wise families and site-local products, 32^3x64 sites (P: 1/8 of the sites)",
                    "unit": "site-updates/s", "value": res["F3_D_vpeq_c_times_D"]["site_updates_per_s"], "ops": res})
    elif args.workload == "fields":
        # the widened families: random fills, global P reductions / sums,
        # gamma and antihermitian maps, N-colour element-wise (nc = 4), the
        # real / complex field library; 32^3x64 sites (P: 1/8 of the sites)
        n = 32 * 32 * 32 * 64
        res = {}
        st = torch.zeros(n, 11, dtype=torch.int32, device="cuda")
        seeds = torch.arange(n, dtype=torch.int32, device="cuda")
        L.QLA_S_veq_seed_i_I(V(st), 2024, V(seeds), n)
        v6 = torch.empty(n, 6, device="cuda")
        d = torch.randn(n, 24, device="cuda")
        d2 = torch.empty_like(d)
        m = torch.randn(n, 18, device="cuda")
        m2 = torch.empty_like(m)
        ps = torch.randn(n // 8, 288, device="cuda")
        ps2 = torch.randn(n // 8, 288, device="cuda")
        red = torch.zeros(288, dtype=torch.float64, device="cuda")
        d4 = torch.randn(n, 32, device="cuda")
        d4b = torch.randn(n, 32, device="cuda")
        cs = torch.tensor([0.3, -0.7], device="cuda")
        ra, rb = torch.rand(n, device="cuda") + 0.5, torch.randn(n, device="cuda")
        ca, cb, cc = torch.randn(n, 2, device="cuda"), torch.randn(n, 2, device="cuda"), torch.empty(n, 2, device="cuda")
        rr = torch.empty(n, device="cuda")
        table = [("QLA_F3_V_veq_gaussian_S", lambda: L.QLA_F3_V_veq_gaussian_S(V(v6), V(st), n), n, 24 + 88),
                 ("QLA_F3_p_veq_sum_P", lambda: L.QLA_F3_p_veq_sum_P(V(red), V(ps), n // 8), n // 8, 1152),
                 ("QLA_F3_c_veq_P_dot_P", lambda: L.QLA_F3_c_veq_P_dot_P(V(red), V(ps), V(ps2), n // 8), n // 8, 2304),
                 ("QLA_F3_D_veq_gamma_times_D", lambda: L.QLA_F3_D_veq_gamma_times_D(V(d2), V(d), 5, n), n, 192),
                 ("QLA_F3_M_veq_antiherm_M", lambda: L.QLA_F3_M_veq_antiherm_M(V(m2), V(m), n), n, 144),
                 ("QLA_FN_D_vpeq_c_times_D(nc=4)", lambda: L.QLA_FN_D_vpeq_c_times_D(4, V(d4), V(cs), V(d4b), n), n, 384),
                 ("QLA_F_R_veq_sin_R", lambda: L.QLA_F_R_veq_sin_R(V(rr), V(rb), n), n, 8),
                 ("QLA_F_C_veq_C_times_C", lambda: L.QLA_F_C_veq_C_times_C(V(cc), V(ca), V(cb), n), n, 24),
                 ("QLA_F_r_veq_R_dot_R", lambda: L.QLA_F_r_veq_R_dot_R(V(red), V(ra), V(rb), n), n, 8)]
        for nm, call, nn, nb in table:
            ms = _events_time(torch, stream, call, reps)
            gbs = nb * nn / (ms / 1e3) / 1e9
            res[nm] = {"site_updates_per_s": nn / (ms / 1e3), "us": 1e3 * ms, "gbs": gbs, "hbm_frac": gbs / peak}
        qla.check("fields")
        out.update({"metric": "widened families (random fills, P reductions, gamma, N-colour, real/complex fields), "
                              "32^3x64 sites (P: 1/8 of the sites)",
                    "unit": "site-updates/s", "value": res["QLA_F3_D_veq_gamma_times_D"]["site_updates_per_s"],
                    "ops": res})
    elif args.workload == "config1":
        n = 16 ** 4
        res = {}
        for pc, dt in (("F3", torch.float32), ("D3", torch.float64)):
            a = torch.randn(n, 18, device="cuda", dtype=dt)
            b = torch.randn(n, 6, device="cuda", dtype=dt)
            r = torch.empty(n, 6, device="cuda", dtype=dt)
            o = torch.zeros(1, dtype=torch.float64, device="cuda")
            rp = "DF3" if pc == "F3" else "D3"
            for nm, fn in (("V_veq_M_times_V", lambda: getattr(L, f"QLA_{pc}_V_veq_M_times_V")(V(r), V(a), V(b), n)),
                           ("V_veq_Ma_times_V", lambda: getattr(L, f"QLA_{pc}_V_veq_Ma_times_V")(V(r), V(a), V(b), n)),
                           ("r_veq_norm2_V", lambda: getattr(L, f"QLA_{rp}_r_veq_norm2_V")(V(o), V(b), n))):
                g = torch.cuda.CUDAGraph()
                s2 = torch.cuda.Stream()
                with torch.cuda.stream(s2):
                    qla.set_stream(s2)
                    fn()
                    torch.cuda.synchronize()
                    with torch.cuda.graph(g, stream=s2):
                        for _ in range(1000):
                            fn()
                qla.set_stream(stream)
                ms = _events_time(torch, stream, g.replay, 3)
                res[f"{pc}_{nm}"] = {"us_per_call": ms, "site_updates_per_s": n * 1000 / (ms / 1e3)}
                del g
            qla.check("config1")
        out.update({"metric": "16^4 F3/D3 V_veq_M_times_V, V_veq_Ma_times_V, r_veq_norm2_V (L2-resident, "
                              "CUDA graph of 1000 launches)", "unit": "site-updates/s",
                    "value": res["F3_V_veq_M_times_V"]["site_updates_per_s"], "ops": res,
                    "note": "8 MB working set lives in L2; no HBM fraction is claimed"})
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # smaller cases for profiler captures (the default is the benchmark workload)
    ap.add_argument("--sites", type=int, default=NSITES)
    ap.add_argument("--iters", type=int, default=ITERS)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the reduction accuracy check")
    ap.add_argument("--no-extra", action="store_true",
                    help="leave the config-2 / config-4 figures out of the benchmark line")
    ap.add_argument("--workload", default="cg_chain", choices=["cg_chain", "hop", "batched", "mfunc", "prop", "ewise", "fields", "config1"],
                    help="cg_chain is the benchmark line; the others measure the remaining configurations")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        print("bench.py: warm-up raised to 3 steps", file=sys.stderr)
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.workload != "cg_chain":
        run_workload(args)
    else:
        run_gpu_arm(args)


if __name__ == "__main__":
    main()
