"""Benchmark: one FMM solve (upward, M2L, downward, near field) of N = 4,194,304 uniform
particles, n = 8 (r = 256), leaves at level 7 (2 particles per leaf on average), q ~ U[-1,1].

A "step" is one solve with charges resident in HBM (value) or from pinned host memory with
the result copied back (e2e). The headline mode is the mixed-precision solver; the plain
FP64 solver of the same FMM is timed beside it for the speed-up and error ratio, both
against an FP64 direct sum on 4,096 seeded targets.

N > 1 GPUs: independent replicas (one solve per rank and step; the path does not shard),
timed on the device with the max over ranks.

--impl reference: the reference's own CPU code (oracle/_ref, built from its sources; else
the CPU oracle port) on the host cores, each step a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_FULL = 4_194_304
N_ORDER = 8
MAXLEV = 7
N_TARGETS = 4096
METRIC = "FMM solves/s at N=4,194,304, n=8, depth 7 (1 GPU; err <= 1.2x FP64 required)"
# DRAM bytes of one m2l_tc2_kernel launch per cell of its level, from an ncu capture of the
# level-6 launch of a depth-6 solve in the form the solve makes it (split rows of the down
# projection written; profiles/m2l_tc2_n8_level6_traffic.md); the traffic scales with the
# number of cells (multipoles in, FP64 output and split rows out): 885.2 MB read + 299.2 MB
# written for 262,144 cells.
TC_DRAM_BYTES_PER_CELL = (885159936 + 299155712) / 262144
SMS, MAX_SM_MHZ = 148, 1965.0
# FP64 tensor (DMMA) peak: 128 FP64 flops per clock per SM (profiles/m2l_lead_n8_level5.md)
DMMA_TFLOPS = SMS * 128 * MAX_SM_MHZ * 1e6 / 1e12
# FP32 SIMT peak (an FMA as two flops per lane, 128 lanes per SM)
FP32_TFLOPS = SMS * 256 * MAX_SM_MHZ * 1e6 / 1e12
# Near-field roof: min(FP32 issue / 7 FP32 operations per pair, reciprocal
# square roots at 16 per clock per SM), in pairs/s at the maximum SM clock
P2P_ROOF_PAIRS = min(SMS * 128 * MAX_SM_MHZ * 1e6 / 7, SMS * 16 * MAX_SM_MHZ * 1e6)


def morton_to_grid(m, level):
    m = np.asarray(m, np.int64)
    ix, iy, iz = (np.zeros_like(m) for _ in range(3))
    for b in range(level):
        t = (m >> (3 * b)) & 7
        ix |= ((t >> 2) & 1) << b
        iy |= ((t >> 1) & 1) << b
        iz |= (t & 1) << b
    return ix, iy, iz


def leaf_counts(x, maxlev, L=1.0):
    """Particles per leaf on the (2^maxlev)^3 grid, from the library's own leaf sort."""
    import ctypes as C
    from bbfmm_b200 import _lib
    x = np.ascontiguousarray(x, np.float64)
    N = x.shape[0]
    perm = np.zeros(N, np.int32)
    ls = np.zeros(8 ** maxlev + 1, np.int32)
    _lib.check(_lib.lib().bbfmm_b200_sort_particles(N, 0, C.c_void_p(x.ctypes.data), L, maxlev,
                                                    perm.ctypes.data_as(C.POINTER(C.c_int)),
                                                    ls.ctypes.data_as(C.POINTER(C.c_int))))
    m = 2 ** maxlev
    g = np.zeros((m, m, m), np.int64)
    ix, iy, iz = morton_to_grid(np.arange(8 ** maxlev), maxlev)
    g[ix, iy, iz] = np.diff(ls)
    return g


def near_pairs(counts):
    """Pair evaluations of the near field, exact from the tree: sum_A n_A sum_{B in N(A)} n_B
    over the leaves and their <= 27 neighbours (anotherNearField.c:326-336; self pairs, which
    the kernels skip, included)."""
    m = counts.shape[0]
    p = np.pad(counts, 1)
    nb = sum(p[1 + dx:1 + dx + m, 1 + dy:1 + dy + m, 1 + dz:1 + dz + m]
             for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1))
    return int((counts * nb).sum())


def pass_bytes(n, maxlev, N, nonempty, mixed):
    """Algorithmic HBM bytes of the passes of one solve (FP64 node values, 8 B each):
    P2M reads the particles (32 B) and writes the leaves' n^3 values (plus their BF16 hi/lo
    split in the mixed mode); M2M reads 8 children and writes the parent per parent cell;
    L2L reads the parent and reads and writes the 8 children; L2P reads the n^3 values of the
    non-empty leaves and the particles and writes phi."""
    n3b = n ** 3 * 8
    leaves = 8 ** maxlev
    par = sum(8 ** l for l in range(2, maxlev))  # parents of levels 3 .. maxlev
    return {"p2m": 32 * N + leaves * n3b + (leaves * n ** 3 * 4 if mixed else 0),
            "m2m": par * (8 * n3b + n3b),
            "l2l": par * (n3b + 2 * 8 * n3b),
            "l2p": nonempty * n3b + 40 * N}


def interactions_per_level(level: int) -> int:
    """Exact number of M2L (target, source) pairs at a level of the full uniform tree."""
    m = 2 ** level
    tot = 0
    for c in range(8):
        b = ((c >> 2) & 1, (c >> 1) & 1, c & 1)
        for vx in range(-3, 4):
            for vy in range(-3, 4):
                for vz in range(-3, 4):
                    if max(abs(vx), abs(vy), abs(vz)) <= 1:
                        continue
                    v = (vx, vy, vz)
                    if any(v[a] < -2 - b[a] or v[a] > 3 - b[a] for a in range(3)):
                        continue
                    cnt = 1
                    for a in range(3):
                        t = np.arange(b[a], m, 2)
                        cnt *= int(((t + v[a] >= 0) & (t + v[a] < m)).sum())
                    tot += cnt
    return tot


class ClockSampler:
    """nvidia-smi sampling during the timed region (SM clock, max clock, throttle reasons)."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_inputs(N, seed):
    rng = np.random.default_rng(seed)
    x = rng.random((N, 3)) - 0.5      # [0,1)^3 shifted onto the origin-centred root cell
    q = rng.uniform(-1.0, 1.0, N)
    return x, q


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), d.get("bf16_tflops_sustained", 1400.0), "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


# ------------------------------------------------------------------ reference arm
def reference_sample(N_sample, maxlev_sample, reps=1, n=N_ORDER):
    """Time the reference's CPU FMM (oracle/_ref) on a sample with the same particles per
    leaf as the full workload; returns (seconds per sample solve, cores, kind)."""
    from oracle.oracle import Oracle, Reference, reference_available
    from bbfmm_b200 import operators as ops
    x, q = make_inputs(N_sample, 99)
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    if reference_available("d"):
        ref = Reference("d")
        d = os.path.join(ops.default_cache_dir(), "ref")
        kp, up = ops.operator_file_names(n, False)
        kp, up = os.path.join(d, kp), os.path.join(d, up)
        if not (os.path.exists(kp) and os.path.exists(up)):
            _, U, E = ops.load_operators(n, False)
            ops.write_operator_files(d, n, U, E, False)
        ref.fmm(x, q, n, maxlev_sample, kp, up)  # warm (file cache, page faults)
        t0 = time.perf_counter()
        for _ in range(reps):
            ref.fmm(x, q, n, maxlev_sample, kp, up)
        return (time.perf_counter() - t0) / reps, cores, "reference"
    _, U, E = ops.load_operators(n, False)
    orc = Oracle("d")
    t0 = time.perf_counter()
    for _ in range(reps):
        orc.fmm(x, q, n, maxlev_sample, U, E)
    return (time.perf_counter() - t0) / reps, 1, "port"


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    # bounded sample: same leaf density (2 per leaf) at level 4 -> 8,192 particles
    Ns, ls = 8192, 4
    times = []
    for i in range(args.warmup + args.steps):
        t, cores, kind = reference_sample(Ns, ls)
        if i >= args.warmup:
            times.append(t)
    t = float(np.mean(times))
    value = (1.0 / t) * (Ns / N_FULL)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solve/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "bbFMM Laplace 1/r, N=4,194,304 uniform, n=8, maxlev 7", "sample_N": Ns,
                       "sample_maxlev": ls},
            "cpu_baseline": {"value": value, "unit": "solve/s", "cores": cores, "kind": kind,
                             "sample": f"one reference CPU solve of N={Ns}, n=8, maxlev {ls} (2 particles/leaf) "
                                       f"per step, scaled by {Ns}/{N_FULL}"},
            "e2e": {"value": value, "unit": "solve/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ other workloads
def _device_time(fn, steps, stream=None):
    """Mean device time (s) of fn() over `steps` calls, CUDA events on `stream` (default:
    torch's current stream), synchronised on both sides."""
    import torch
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / 1e3 / steps


def clustered_inputs(N, seed, clusters=8, sigma=0.05, lo=0.15, hi=0.85):
    """Positions from isotropic Gaussian clusters (centres U[lo, hi]^3) clipped to [0,1)^3 and
    shifted onto the origin-centred root cell; charges U[-1, 1]; loss weights N(0, 1)."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(lo, hi, (clusters, 3))
    x = c[rng.integers(0, clusters, N)] + sigma * rng.standard_normal((N, 3))
    x = np.clip(x, 0.0, np.nextafter(1.0, 0.0)) - 0.5
    return x, rng.uniform(-1.0, 1.0, N), rng.standard_normal(N)


def run_uniform_32k(args):
    """N = 32,768 uniform, n = 4, maxlev 4, FP64: every potential against the FP64 direct sum,
    the reference CPU code on the same input beside it."""
    import torch
    from bbfmm_b200 import Solver
    from bbfmm_b200.fmm import direct
    N, n, lev = 32768, 4, 4
    x, q = make_inputs(N, 1)
    sol = Solver(n, lev, 1.0, mode="d")
    sol.set_particles(x)
    qd = torch.as_tensor(q, device="cuda")
    out = torch.empty_like(qd)
    stream = torch.cuda.ExternalStream(sol.stream)
    for _ in range(args.warmup):
        sol.solve(qd, out=out)
    t = _device_time(lambda: sol.solve(qd, out=out), args.steps, stream)
    qh = torch.as_tensor(q).pin_memory().numpy()
    for _ in range(2):
        sol.solve_host(qh)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ph = sol.solve_host(qh)
    t_e2e = (time.perf_counter() - t0) / args.steps
    sol.set_timing(True)
    sol.solve(qd, out=out)
    torch.cuda.synchronize()
    stages, launches = sol.stage_times()
    ex = direct(torch.as_tensor(x, device="cuda"), qd, torch.arange(N, dtype=torch.int32, device="cuda")).cpu().numpy()
    err = float(np.linalg.norm(ph - ex) / np.linalg.norm(ex))
    t_ref, cores, kind = reference_sample(N, lev, reps=3, n=n) if not args.no_cpu_baseline else (None, 0, None)
    line = {"metric": "FMM solves/s at N=32,768 uniform, n=4, depth 4, FP64", "value": 1.0 / t, "unit": "solve/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded uniform [0,1)^3, q~U[-1,1])",
            "config": {"workload": "bbFMM Laplace 1/r, N=32,768 uniform, n=4 (r=32), maxlev 4", "N": N, "n": n,
                       "maxlev": lev, "mode": "d", "l2": "working set fits in L2 (small configuration)"},
            "err_vs_fp64_direct_all_targets": err, "stages_ms": stages, "gpu_launches": launches * args.steps,
            "e2e": {"value": 1.0 / t_e2e, "unit": "solve/s", "h2d_bytes_per_step": 8 * N, "d2h_bytes_per_step": 8 * N},
            "cpu_baseline": None if t_ref is None else {
                "value": 1.0 / t_ref, "unit": "solve/s", "cores": cores, "kind": kind,
                "sample": f"the whole workload (N={N}, n={n}, maxlev {lev}), mean of 3 solves"}}
    print(json.dumps(line), flush=True)
    return 0


def run_uniform_4m_variants(args):
    """The other precision/order forms of the 4M-particle uniform workload (N = 4,194,304,
    maxlev 7, seeded like the headline line): n in {4, 8} x modes d / s / mixed, and the FP32
    tolerance-rank form (SVD cut at 1e-5), each timed over `steps` device-resident solves and
    checked against the FP64 direct sum on the headline's 4,096 seeded targets; the
    reference CPU code for n = 4 on a bounded sample beside them."""
    import torch
    from bbfmm_b200 import Solver
    from bbfmm_b200.fmm import direct
    N, lev = args.N, args.maxlev
    x, q = make_inputs(N, 2)
    targets = np.random.default_rng(1234).choice(N, N_TARGETS, replace=False).astype(np.int32)
    dref = direct(torch.as_tensor(x, device="cuda"), torch.as_tensor(q, device="cuda"),
                  torch.as_tensor(targets, device="cuda")).cpu().numpy()
    forms = [(4, "d", None), (4, "s", None), (4, "mixed", None), (8, "d", None), (8, "s", None),
             (8, "mixed", None), (8, "s", 1e-5)]
    out = []
    for n, mode, tol in forms:
        sol = Solver(n, lev, 1.0, mode=mode, tol=tol)
        sol.set_particles(x)
        dt = torch.float32 if mode == "s" else torch.float64
        qd = torch.as_tensor(q, dtype=dt, device="cuda")
        ph = torch.empty_like(qd)
        stream = torch.cuda.ExternalStream(sol.stream)
        steps = args.steps if n == 4 or mode == "mixed" else min(args.steps, 2)
        sol.solve(qd, out=ph)
        t = _device_time(lambda: sol.solve(qd, out=ph), steps, stream)
        a = ph.double().cpu().numpy()[targets]
        err = float(np.sqrt(((a - dref) ** 2).sum() / (dref ** 2).sum()))
        out.append({"n": n, "mode": mode, "tol": tol, "rank": sol.rank if tol else n ** 3 // 2,
                    "s_per_solve": t, "steps": steps, "err_vs_fp64_direct": err})
        sol.close()
        del sol
        torch.cuda.empty_cache()
    base = {(o["n"], o["mode"]): o for o in out if o["tol"] is None}
    for o in out:
        d = base.get((o["n"], "d"))
        o["speedup_vs_fp64_gpu"] = d["s_per_solve"] / o["s_per_solve"] if d else None
        o["err_ratio_vs_fp64_gpu"] = o["err_vs_fp64_direct"] / d["err_vs_fp64_direct"] if d else None
    t_ref, cores, kind = (reference_sample(65536, 5, n=4) if not args.no_cpu_baseline else (None, 0, None))
    head = base[(4, "mixed")]
    line = {"metric": "FMM solves/s at N=4,194,304 uniform, depth 7: n = 4 / 8, FP64 / FP32 / mixed",
            "value": 1.0 / head["s_per_solve"], "unit": "solve/s", "n_gpus": 1, "steps": args.steps,
            "warmup": 1, "ms_per_step": head["s_per_solve"] * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded uniform [0,1)^3, q~U[-1,1])",
            "config": {"workload": "bbFMM Laplace 1/r, N=4,194,304 uniform, maxlev 7, order and precision forms",
                       "N": N, "maxlev": lev, "headline_form": "n=4 mixed"},
            "forms": out,
            "cpu_baseline": None if t_ref is None else {
                "value": 1.0 / (t_ref * N / 65536), "unit": "solve/s", "cores": cores, "kind": kind,
                "sample": "one CPU solve of N=65536, n=4, maxlev 5 (2 particles/leaf), scaled by N"}}
    print(json.dumps(line), flush=True)
    return 0


def _gradient_case(mode, x, q, w, args):
    """Forward and forward + backward of L = sum_i w_i phi_i in one precision mode: timings,
    bytes kept for the backward, and the gradients (of the last save mode)."""
    import torch
    from bbfmm_b200 import Solver
    from bbfmm_b200.autograd import fmm_phi
    free0 = torch.cuda.mem_get_info()[0]
    sol = Solver(8, 6, 1.0, mode=mode)
    sol.set_particles(x)
    dt = sol.dtype
    qd = torch.as_tensor(q, dtype=dt, device="cuda")
    xd = torch.as_tensor(x, dtype=dt, device="cuda")
    wd = torch.as_tensor(w, dtype=dt, device="cuda")
    out = torch.empty_like(qd)
    stream = torch.cuda.ExternalStream(sol.stream)
    for _ in range(args.warmup):
        sol.solve(qd, out=out)
    torch.cuda.synchronize()
    solver_bytes = free0 - torch.cuda.mem_get_info()[0]
    t_fwd = _device_time(lambda: sol.solve(qd, out=out), args.steps, stream)
    res = {}
    for save in ("fields", "recompute"):
        def fwd_bwd():
            qt = qd.clone().requires_grad_(True)
            xt = xd.clone().requires_grad_(True)
            L = (wd * fmm_phi(sol, qt, xt, save=save)).sum()
            L.backward()
            return qt.grad, xt.grad
        for _ in range(args.warmup):
            fwd_bwd()
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats()
        base = torch.cuda.memory_allocated()
        gq, gx = fwd_bwd()
        torch.cuda.synchronize()
        peak = torch.cuda.max_memory_allocated() - base
        t = _device_time(fwd_bwd, args.steps)
        # bytes the forward keeps for the backward
        qt = qd.clone().requires_grad_(True)
        xt = xd.clone().requires_grad_(True)
        m0 = torch.cuda.memory_allocated()
        y = fmm_phi(sol, qt, xt, save=save)
        torch.cuda.synchronize()
        kept = torch.cuda.memory_allocated() - m0 - y.numel() * y.element_size()
        del y
        res[save] = {"fwd_bwd_ms": t * 1e3, "fwd_bwd_over_fwd": t / t_fwd, "saved_bytes": int(kept),
                     "peak_torch_bytes_fwd_bwd": int(peak)}
        grads = (gq.double(), gx.double())
    sol.close()
    return {"forward_ms": t_fwd * 1e3, "save_modes": res, "solver_device_bytes": int(solver_bytes)}, grads


def run_gradient_1m(args):
    """N = 1,048,576 from 8 Gaussian clusters, n = 8, maxlev 6: forward, and forward +
    backward of L = sum_i w_i phi_i through fmm_phi with both ways of keeping the backward's
    inputs (fields checkpointed, or recomputed), their saved bytes, and the gradients against
    the FP64 direct-sum analytic gradient on 4,096 targets; in FP32 (the configuration's
    forward precision, the line's value) and in the mixed mode."""
    import torch
    from bbfmm_b200.fmm import direct_field
    N, n, lev = 1_048_576, 8, 6
    x, q, w = clustered_inputs(N, 11)
    targets = np.random.default_rng(1234).choice(N, N_TARGETS, replace=False).astype(np.int32)
    td = torch.as_tensor(targets, device="cuda")
    x64, q64, w64 = (torch.as_tensor(a, device="cuda") for a in (x, q, w))
    p1, f1 = direct_field(x64, q64, td)
    p2, f2 = direct_field(x64, w64 * q64, td)
    wt, qt_ = w64[td.long()], q64[td.long()]
    dq = wt * p1 + p2
    dx = qt_[:, None] * (wt[:, None] * f1 + f2)
    modes = {}
    for mode in (["d"] if args.mode == "d" else ["s", "mixed"]):
        r, (gq, gx) = _gradient_case(mode, x, q, w, args)
        r["grad_err_vs_fp64_direct"] = {
            "dq": float(torch.linalg.norm(gq[td.long()] - dq) / torch.linalg.norm(dq)),
            "dx": float(torch.linalg.norm(gx[td.long()] - dx) / torch.linalg.norm(dx)), "n_targets": N_TARGETS}
        modes[mode] = r
        torch.cuda.empty_cache()
    head_mode = "d" if args.mode == "d" else "s"
    head = modes[head_mode]
    line = {"metric": "forward+backward of sum(w*phi) at N=1,048,576 clustered, n=8, depth 6",
            "value": 1.0 / (head["save_modes"]["fields"]["fwd_bwd_ms"] / 1e3), "unit": "fwd+bwd/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["save_modes"]["fields"]["fwd_bwd_ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"d": "f64", "s": "f32"}[head_mode],
            "data": "synthetic (seeded 8-Gaussian mixture, sigma 0.05)",
            "config": {"workload": "bbFMM Laplace 1/r gradients, N=1,048,576 clustered, n=8, maxlev 6", "N": N,
                       "n": n, "maxlev": lev, "mode": head_mode},
            "modes": modes}
    print(json.dumps(line), flush=True)
    return 0


def clustered_16m_inputs(seed=3, N=16_777_216):
    """Half uniform in the unit cube, half from 16 isotropic Gaussian clusters (centres
    U[0.1, 0.9]^3, sigma 0.03, clipped to the cube), shifted onto the origin-centred root
    cell; charges N(0, 1)."""
    rng = np.random.default_rng(seed)
    nu = N // 2
    c = rng.uniform(0.1, 0.9, (16, 3))
    xc = c[rng.integers(0, 16, N - nu)] + 0.03 * rng.standard_normal((N - nu, 3))
    x = np.concatenate([rng.random((nu, 3)), np.clip(xc, 0.0, np.nextafter(1.0, 0.0))]) - 0.5
    return x, rng.standard_normal(N)


def run_clustered_16m(args):
    """N = 16,777,216 clustered (50% uniform + 50% in 16 Gaussians), n = 8, depth 8: the M2L
    precisions side by side -- FP64 leading block + 3xBF16 (the mixed mode), 3xBF16 alone,
    plain BF16 (one product), FP32 and FP64 -- each timed and compared with the FP64 direct
    sum on 8,192 sampled targets (relative L2 and max error / max |phi|). The leaf level runs
    in slabs (its n^3 node arrays would take 69 GB each in FP64). The default mixed mode uses
    the adaptive product map (three split-BF16 products only where one would not do)."""
    import torch
    from bbfmm_b200 import Solver
    from bbfmm_b200.fmm import direct
    N, n, lev = 16_777_216, 8, 8
    x, q = clustered_16m_inputs()
    targets = np.random.default_rng(4321).choice(N, 8192, replace=False).astype(np.int32)
    ref = direct(torch.as_tensor(x, device="cuda"), torch.as_tensor(q, device="cuda"),
                 torch.as_tensor(targets, device="cuda")).cpu().numpy()
    variants = [("fp64 lead + adaptive bf16", "mixed", 16, 0), ("fp64 lead + 3xbf16", "mixed", 16, 3),
                ("3xbf16", "mixed", 0, 3), ("1xbf16", "mixed", 0, 1), ("fp32", "s", 0, 3), ("fp64", "d", 0, 3)]
    res = {}
    for name, mode, lead, nprod in variants:
        free0 = torch.cuda.mem_get_info()[0]
        sol = Solver(n, lev, 1.0, mode=mode, lead=lead if lead else 0)
        if mode == "mixed":
            sol.set_tc_products(nprod)
        sol.set_particles(x)
        dt = sol.dtype
        qd = torch.as_tensor(q, dtype=dt, device="cuda")
        out = torch.empty_like(qd)
        stream = torch.cuda.ExternalStream(sol.stream)
        sol.solve(qd, out=out)
        torch.cuda.synchronize()
        used = free0 - torch.cuda.mem_get_info()[0]
        steps = args.steps if mode == "mixed" else 1
        with ClockSampler(0) as clk:
            t = _device_time(lambda: sol.solve(qd, out=out), steps, stream)
        sol.set_timing(True)
        sol.solve(qd, out=out)
        torch.cuda.synchronize()
        stages, _ = sol.stage_times()
        sol.set_timing(False)
        phi = out.double().cpu().numpy()[targets]
        res[name] = {"mode": mode, "lead": lead, "products": nprod, "s_per_solve": t,
                     "err_rel_l2": float(np.linalg.norm(phi - ref) / np.linalg.norm(ref)),
                     "err_max_over_max_abs": float(np.abs(phi - ref).max() / np.abs(ref).max()),
                     "device_bytes": int(used), "stages_ms": stages, "clocks": clk.summary()}
        sol.close()
        del qd, out
        torch.cuda.empty_cache()
    head = res["fp64 lead + adaptive bf16"]
    line = {"metric": "FMM solves/s at N=16,777,216 clustered, n=8, depth 8", "value": 1.0 / head["s_per_solve"],
            "unit": "solve/s", "n_gpus": 1, "steps": args.steps, "warmup": 1,
            "ms_per_step": head["s_per_solve"] * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16x3+f64",
            "data": "synthetic (seeded; 50% uniform, 50% in 16 Gaussians sigma 0.03; q ~ N(0,1))",
            "config": {"workload": "bbFMM Laplace 1/r, N=16,777,216 clustered, n=8 (r=256), maxlev 8", "N": N,
                       "n": n, "maxlev": lev, "n_targets": 8192},
            "variants": res,
            "err_ratio_vs_fp64": head["err_rel_l2"] / res["fp64"]["err_rel_l2"],
            "speedup_vs_fp64": res["fp64"]["s_per_solve"] / head["s_per_solve"]}
    print(json.dumps(line), flush=True)
    return 0


def run_clustered_16m_adaptive(args):
    """The N = 16,777,216 clustered input (configuration 3) through the two-level adaptive
    solver (coarse depth 6 for the uniform half, depth-8 refinement of the leaves holding more
    than 256 particles) beside the uniform mixed solve of depth 8, both against the FP64 direct
    sum on the same 8,192 targets."""
    import torch
    from bbfmm_b200 import AdaptiveSolver, Solver
    from bbfmm_b200.fmm import direct
    N = 16_777_216
    x, q = clustered_16m_inputs()
    targets = np.random.default_rng(4321).choice(N, 8192, replace=False).astype(np.int32)
    ref = direct(torch.as_tensor(x, device="cuda"), torch.as_tensor(q, device="cuda"),
                 torch.as_tensor(targets, device="cuda")).cpu().numpy()
    qd = torch.as_tensor(q, device="cuda")
    res = {}
    for name in ("adaptive", "uniform"):
        t0 = time.perf_counter()
        if name == "adaptive":
            s = AdaptiveSolver(8, 6, 8, mode="mixed", cap=256)
        else:
            s = Solver(8, 8, 1.0, mode="mixed")
        s.set_particles(x)
        t_setup = time.perf_counter() - t0
        out = s.solve(qd)
        torch.cuda.synchronize()
        with ClockSampler(0) as clk:
            t = _device_time(lambda: s.solve(qd, out=out), args.steps)
        phi = out.double().cpu().numpy()[targets]
        r = {"s_per_solve": t, "setup_s": t_setup, "clocks": clk.summary(),
             "err_rel_l2": float(np.linalg.norm(phi - ref) / np.linalg.norm(ref))}
        if name == "adaptive":
            r.update({"heavy_leaves_depth6": s.heavy_leaves, "refined_particles": s.fine_particles})
        res[name] = r
        s.close()
        del s, out
        torch.cuda.empty_cache()
    head = res["adaptive"]
    line = {"metric": "FMM solves/s at N=16,777,216 clustered, n=8: two-level adaptive (depth 6 + 8) vs uniform depth 8",
            "value": 1.0 / head["s_per_solve"], "unit": "solve/s", "n_gpus": 1, "steps": args.steps,
            "warmup": 1, "ms_per_step": head["s_per_solve"] * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16x3+f64",
            "data": "synthetic (seeded; 50% uniform, 50% in 16 Gaussians sigma 0.03; q ~ N(0,1))",
            "config": {"workload": "bbFMM Laplace 1/r, N=16,777,216 clustered, n=8, adaptive depth 6 + 8", "N": N,
                       "n": 8, "n_targets": 8192, "cap": 256},
            "variants": res, "speedup_vs_uniform": res["uniform"]["s_per_solve"] / head["s_per_solve"],
            "err_ratio_vs_uniform": head["err_rel_l2"] / res["uniform"]["err_rel_l2"]}
    print(json.dumps(line), flush=True)
    return 0


def batch_sets(seed=5, nsets=256):
    """256 independent sets: N log-uniform in [4096, 262144], half uniform in the unit cube and
    half from 4 Gaussian clusters (sigma 0.04, centres U[0.1, 0.9]^3, clipped), n = 4 or 8 at
    random, depth round(log8(N / 32)) (about 32 particles per leaf); charges U[-1, 1]."""
    from bbfmm_b200 import batch_depth
    rng = np.random.default_rng(seed)
    sets = []
    for k in range(nsets):
        N = int(round(np.exp(rng.uniform(np.log(4096), np.log(262144)))))
        if k % 2 == 0:
            x = rng.random((N, 3))
        else:
            c = rng.uniform(0.1, 0.9, (4, 3))
            x = np.clip(c[rng.integers(0, 4, N)] + 0.04 * rng.standard_normal((N, 3)), 0.0, np.nextafter(1.0, 0.0))
        n = int(rng.choice([4, 8]))
        sets.append((x - 0.5, n, batch_depth(N)))
    q = rng.uniform(-1.0, 1.0, sum(len(x) for x, _, _ in sets))
    return sets, q


def run_batch_256(args, adaptive=False):
    """256 uneven sets in one batch (stacked per (n, depth), one launch per pass per group,
    the groups as parallel branches of one CUDA graph), after the autotuner; per-set error
    against the FP64 direct sum on 512 sampled targets per set. adaptive: the same sets through
    AdaptiveBatch (leaves of more than 256 particles refined by two levels in a second batch)."""
    import torch
    import torch.distributed as dist
    from bbfmm_b200 import AdaptiveBatch, Batch, set_cost, shard_sets
    from bbfmm_b200.fmm import direct
    mode = args.mode
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    all_sets, all_q = batch_sets()
    # N GPUs: the sets are split by a cost model (no collective on the data path)
    offs_all = np.concatenate([[0], np.cumsum([len(x) for x, _, _ in all_sets])])
    mine = shard_sets([set_cost(len(x), n, lev) for x, n, lev in all_sets], world)[rank]
    sets = [all_sets[i] for i in mine]
    q = np.concatenate([all_q[offs_all[i]:offs_all[i + 1]] for i in mine]) if mine else np.zeros(0)
    t0 = time.perf_counter()
    b = AdaptiveBatch(sets, mode=mode, cap=256, device=local) if adaptive else Batch(sets, mode=mode, device=local)
    t_setup = time.perf_counter() - t0
    dt = torch.float32 if mode == "s" else torch.float64
    qd = torch.as_tensor(q, dtype=dt, device="cuda")
    out = torch.empty_like(qd)
    t0 = time.perf_counter()
    if adaptive:
        b.autotune(qd)
        groups = b.coarse.groups() + (b.refined.groups() if b.refined is not None else [])
    else:
        groups = b.autotune(qd)
    t_tune = time.perf_counter() - t0
    # the adaptive batch's solve spans two batch streams and the caller's: time on the caller's
    stream = None if adaptive else torch.cuda.ExternalStream(b.stream)
    for _ in range(args.warmup):
        b.solve(qd, out=out, graph=True)
    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    barrier()
    # the adaptive batch: the submission its autotune chose (graphs or launches)
    sub = b.graph if adaptive else True
    with ClockSampler(local) as clk:
        t_graph = max_over_ranks(_device_time(lambda: b.solve(qd, out=out, graph=sub), args.steps, stream))
    barrier()
    t_eager = max_over_ranks(_device_time(lambda: b.solve(qd, out=out, graph=False), args.steps, stream))
    t_replay = max_over_ranks(_device_time(lambda: b.solve(qd, out=out, graph=True), args.steps, stream))
    if adaptive:  # the coarse groups, then the refined ones on the charges the last solve gathered
        group_ms = [b.coarse.group_stage_times(qd, g) for g in range(len(b.coarse.groups()))]
        if b.refined is not None:
            group_ms += [b.refined.group_stage_times(b.q_ref, g) for g in range(len(b.refined.groups()))]
    else:
        group_ms = [b.group_stage_times(qd, g) for g in range(len(groups))]
    phi = out.double().cpu().numpy()
    # per-set error on 512 sampled targets
    rng = np.random.default_rng(77)
    errs = []
    for k, (x, n, lev) in enumerate(sets):
        a, e = int(b.offsets[k]), int(b.offsets[k + 1])
        t = rng.choice(e - a, min(512, e - a), replace=False).astype(np.int32)
        ref = direct(torch.as_tensor(x, device="cuda"), torch.as_tensor(q[a:e], device="cuda"),
                     torch.as_tensor(t, device="cuda")).cpu().numpy()
        errs.append(float(np.linalg.norm(phi[a:e][t] - ref) / np.linalg.norm(ref)))
    if world > 1:
        gathered = [None] * world
        dist.all_gather_object(gathered, (errs, [n for _, n, _ in sets]))
        errs = [e for g in gathered for e in g[0]]
        ns = np.array([n for g in gathered for n in g[1]])
    else:
        ns = np.array([n for _, n, _ in sets])
    errs = np.array(errs)
    Ntot = int(offs_all[-1])
    qh = torch.as_tensor(q, dtype=dt).pin_memory()
    ph = torch.empty_like(qh).pin_memory()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        qd.copy_(qh, non_blocking=True)
        b.solve(qd, out=out, graph=sub)
        ph.copy_(out, non_blocking=True)
    torch.cuda.synchronize()
    t_e2e = max_over_ranks((time.perf_counter() - t0) / args.steps)
    t_setup_dev = None
    if not adaptive:  # the same batch from positions already on the device (trees sorted there)
        dsets = [(torch.as_tensor(x, dtype=dt, device="cuda"), n, lev) for x, n, lev in sets]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        bd = Batch(dsets, mode=mode, device=local)
        t_setup_dev = time.perf_counter() - t0
        bd.close()
        del dsets
    cpu = None
    if not args.no_cpu_baseline and rank == 0:
        # the reference CPU code on 4 of the sets (one per (n, depth) seen first), scaled by particles
        t_ref, n_ref, kinds = 0.0, 0, set()
        for (x, n, lev) in sets:
            if (n, lev) in kinds or len(kinds) >= 4:
                continue
            kinds.add((n, lev))
            from oracle.oracle import Reference, reference_available
            if not reference_available("d"):
                break
            tt, cores, kind = reference_sample_xq(x, q[:len(x)], n, lev)
            t_ref += tt
            n_ref += len(x)
        if n_ref:
            cpu = {"value": (n_ref / t_ref) / Ntot, "unit": "batch/s", "cores": cores, "kind": kind,
                   "sample": f"the reference CPU code on {len(kinds)} of the sets ({n_ref} particles, {t_ref:.2f} s), "
                             f"scaled to the batch's {Ntot} particles"}
    line = {"metric": "batched solves of 256 uneven sets (N log-uniform 4,096..262,144, n in {4,8})"
                      + (", two-level adaptive" if adaptive else ""),
            "value": 1.0 / t_graph, "unit": "batch/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_graph * 1e3, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": {"mixed": "bf16x3+f64", "d": "f64", "s": "f32"}[mode],
            "data": "synthetic (seeded; half uniform, half 4-Gaussian sigma 0.04)",
            "config": {"workload": "256 uneven bbFMM Laplace sets, n in {4,8}, depth round(log8(N/32))",
                       "particles": Ntot, "mode": mode, "parallelism": f"sets sharded over {world} GPU(s)",
                       "groups": [{k: g[k] for k in ("n", "maxlev", "sets", "particles", "p2p_threads",
                                                      "m2l_kind", "m2l_groups")} for g in groups]},
            "particles_per_s": Ntot / t_graph, "eager_ms": t_eager * 1e3, "graph_ms": t_replay * 1e3,
            "submission": "graph" if sub else "launches",
            "graph_nodes": None if adaptive else b.graph_nodes,
            "adaptive": {"heavy_leaves": b.heavy_leaves, "refined_particles": b.refined_particles,
                         "cap": 256, "refine_levels": 2} if adaptive else None,
            "group_stage_ms": group_ms,
            "setup_s": t_setup, "setup_device_trees_s": t_setup_dev, "autotune_s": t_tune,
            "err_vs_fp64_direct": {"median": float(np.median(errs)), "max": float(errs.max()),
                                   "max_n4": float(errs[ns == 4].max()), "max_n8": float(errs[ns == 8].max()),
                                   "targets_per_set": 512},
            "e2e": {"value": 1.0 / t_e2e, "unit": "batch/s", "h2d_bytes_per_step": Ntot * qd.element_size(),
                    "d2h_bytes_per_step": Ntot * qd.element_size()},
            "cpu_baseline": cpu, "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line), flush=True)
    b.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def layout_inputs(N, layout, seed=2):
    """Seeded positions in the origin-centred unit root cell and charges U[-1, 1]: "uniform",
    or "clustered" (4 Gaussian clusters, sigma 0.04, centres U[0.1, 0.9]^3, clipped -- the
    clustered sets of the 256-set batch)."""
    rng = np.random.default_rng(seed)
    if layout == "uniform":
        x = rng.random((N, 3))
    else:
        c = rng.uniform(0.1, 0.9, (4, 3))
        x = np.clip(c[rng.integers(0, 4, N)] + 0.04 * rng.standard_normal((N, 3)), 0.0, np.nextafter(1.0, 0.0))
    return np.ascontiguousarray(x - 0.5), rng.uniform(-1.0, 1.0, N)


def run_near_field(args):
    """The near field alone through the caller-owned entry point bbfmm_b200_near_field (mode
    MIXED; leaf-sorted FP64 particles and leaf offsets on the device), timed per call with CUDA
    events around the call (it builds its work list and synchronises); pairs exact from the tree."""
    import ctypes as C
    import torch
    from bbfmm_b200 import _lib
    N, lev = args.N, args.maxlev
    x, q = layout_inputs(N, args.layout)
    perm = np.zeros(N, np.int32)
    ls = np.zeros(8 ** lev + 1, np.int32)
    L = _lib.lib()
    _lib.check(L.bbfmm_b200_sort_particles(N, 0, C.c_void_p(x.ctypes.data), 1.0, lev,
                                           perm.ctypes.data_as(C.POINTER(C.c_int)),
                                           ls.ctypes.data_as(C.POINTER(C.c_int))))
    dx = torch.as_tensor(np.concatenate([x[perm], q[perm, None]], axis=1), device="cuda")
    dl = torch.as_tensor(ls, device="cuda")
    phi = torch.zeros(N, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def call():
        _lib.check(L.bbfmm_b200_near_field(N, lev, 1.0, C.c_void_p(dx.data_ptr()), C.c_void_p(dl.data_ptr()),
                                           C.c_void_p(phi.data_ptr()), 2, C.c_void_p(stream.cuda_stream)))
    for _ in range(args.warmup):
        call()
    t = _device_time(call, max(args.steps, 1), stream)
    pairs = near_pairs(leaf_counts(x, lev))
    line = {"metric": f"near-field pair evaluations/s, N={N} {args.layout}, depth {lev}",
            "value": pairs / t, "unit": "pair/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 separation + f32 terms", "data": f"synthetic ({args.layout}, seeded)",
            "config": {"workload": "bbfmm_b200_near_field (MIXED)", "N": N, "maxlev": lev, "layout": args.layout},
            "pairs": pairs, "frac_of_roof": pairs / t / P2P_ROOF_PAIRS}
    print(json.dumps(line), flush=True)
    return 0


def run_stages(args):
    """Per-stage device times (CUDA events between stages) of one solver configuration: the
    best of `steps` timed solves after `warmup` plain ones."""
    import torch
    from bbfmm_b200 import Solver
    x, q = layout_inputs(args.N, args.layout)
    s = Solver(N_ORDER, args.maxlev, 1.0, mode=args.mode)
    s.set_particles(x)
    qd = torch.as_tensor(q, dtype=s.dtype, device="cuda")
    out = torch.empty_like(qd)
    for _ in range(args.warmup):
        s.solve(qd, out=out)
    s.set_timing(True)
    best = {}
    for _ in range(max(args.steps, 1)):
        s.solve(qd, out=out)
        torch.cuda.synchronize()
        st, launches = s.stage_times()
        best = {k: min(best.get(k, 1e30), v) for k, v in st.items()}
    line = {"metric": f"stage times of one solve, N={args.N} {args.layout}, n={N_ORDER}, depth {args.maxlev}",
            "value": sum(best.values()), "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sum(best.values()), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": {"mixed": "bf16x3+f64", "d": "f64", "s": "f32"}[args.mode],
            "data": f"synthetic ({args.layout}, seeded)",
            "config": {"workload": "one solve, stage by stage", "N": args.N, "maxlev": args.maxlev, "mode": args.mode,
                       "layout": args.layout},
            "stages_ms": best, "near_pairs": near_pairs(leaf_counts(x, args.maxlev))}
    print(json.dumps(line), flush=True)
    return 0


def reference_sample_xq(x, q, n, lev):
    """Seconds of one reference CPU solve of the given particles (n, depth lev)."""
    from oracle.oracle import Reference
    from bbfmm_b200 import operators as ops
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    ref = Reference("d")
    d = os.path.join(ops.default_cache_dir(), "ref")
    kp, up = ops.operator_file_names(n, False)
    kp, up = os.path.join(d, kp), os.path.join(d, up)
    if not (os.path.exists(kp) and os.path.exists(up)):
        _, U, E = ops.load_operators(n, False)
        ops.write_operator_files(d, n, U, E, False)
    ref.fmm(x, q, n, lev, kp, up)
    t0 = time.perf_counter()
    ref.fmm(x, q, n, lev, kp, up)
    return time.perf_counter() - t0, cores, "reference"


# ------------------------------------------------------------------ our arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="mixed", choices=["mixed", "d", "s"])
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--tol-rank", type=float, default=1e-8,
                    help="also time mixed and plain FP64 with the SVD cut at this relative singular value (0: off)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--N", type=int, default=N_FULL)
    ap.add_argument("--maxlev", type=int, default=MAXLEV)
    ap.add_argument("--workload", default="uniform-4m",
                    choices=["uniform-4m", "uniform-4m-variants", "uniform-32k", "gradient-1m", "batch-256",
                             "clustered-16m", "clustered-16m-adaptive", "batch-256-adaptive", "near-field",
                             "stages"],
                    help="uniform-4m: the headline line; the others measure further configurations")
    ap.add_argument("--layout", default="uniform", choices=["uniform", "clustered"],
                    help="near-field / stages workloads: particle layout")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "uniform-4m-variants":
        return run_uniform_4m_variants(args)
    if args.workload == "uniform-32k":
        return run_uniform_32k(args)
    if args.workload == "gradient-1m":
        return run_gradient_1m(args)
    if args.workload == "batch-256":
        return run_batch_256(args)
    if args.workload == "clustered-16m":
        return run_clustered_16m(args)
    if args.workload == "batch-256-adaptive":
        return run_batch_256(args, adaptive=True)
    if args.workload == "clustered-16m-adaptive":
        return run_clustered_16m_adaptive(args)
    if args.workload == "near-field":
        return run_near_field(args)
    if args.workload == "stages":
        return run_stages(args)

    import torch
    import torch.distributed as dist
    from bbfmm_b200 import Solver
    from bbfmm_b200.fmm import direct
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    N, n, lev = args.N, N_ORDER, args.maxlev
    x, q = make_inputs(N, 2 + rank)
    dt = torch.float32 if args.mode == "s" else torch.float64
    sol = Solver(n, lev, 1.0, mode=args.mode, device=local)
    # tree setup (outside the metric): host build, then the same tree built on the GPU
    t0 = time.perf_counter()
    sol.set_particles(x)
    t_setup_host = time.perf_counter() - t0
    xd = torch.as_tensor(x, dtype=dt, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sol.set_particles(xd)
    torch.cuda.synchronize()
    t_setup_dev = time.perf_counter() - t0
    del xd
    q_dev = torch.as_tensor(q, dtype=dt, device="cuda")
    phi_dev = torch.empty_like(q_dev)
    stream = torch.cuda.ExternalStream(sol.stream)

    def step():
        sol.solve(q_dev, out=phi_dev)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    t_dev = max_over_ranks(ev0.elapsed_time(ev1) / 1e3) / args.steps
    value = world / t_dev

    # end to end through the public host-buffer entry point (pinned host memory)
    q_host = torch.as_tensor(q, dtype=dt).pin_memory().numpy()
    phi_pinned = torch.empty(N, dtype=dt).pin_memory().numpy()
    for _ in range(2):
        sol.solve_host(q_host, out=phi_pinned)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ee0.record(stream)
    for _ in range(args.steps):
        phi_host = sol.solve_host(q_host, out=phi_pinned)
    ee1.record(stream)
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(max(ee0.elapsed_time(ee1) / 1e3, 0.0) / args.steps)
    t_e2e_wall = (time.perf_counter() - t0) / args.steps
    t_e2e = max(t_e2e, max_over_ranks(t_e2e_wall))
    esz = 4 if args.mode == "s" else 8

    # accuracy against the FP64 direct sum on seeded targets
    targets = np.random.default_rng(1234).choice(N, N_TARGETS, replace=False).astype(np.int32)
    xd = torch.as_tensor(x, device="cuda")
    qd64 = torch.as_tensor(q, device="cuda")
    td = torch.as_tensor(targets, device="cuda")
    dref = direct(xd, qd64, td).cpu().numpy()
    phi_mode = phi_dev.double().cpu().numpy()
    def rel(a):
        return float(np.sqrt(((a[targets] - dref) ** 2).sum() / (dref ** 2).sum()))
    err_mode = rel(phi_mode)

    # stage breakdown and the dominant kernel's launch time (CUDA events on the solver stream)
    sol.set_timing(True)
    sol.solve(q_dev, out=phi_dev)
    torch.cuda.synchronize()
    stages, launches = sol.stage_times()
    sol.set_timing(False)
    m2l_ms, lead_ms = sol.time_m2l(lev, reps=3)
    I_leaf = interactions_per_level(lev)
    I_all = sum(interactions_per_level(l) for l in range(2, lev + 1))
    r = n ** 3 // 2
    hbm, bf16, bf16_sus, peak_src = measured_peaks()
    clk_now = clk.summary()
    sm_mhz = clk_now["sm_mhz"] or MAX_SM_MHZ
    # M2L flop counts: 2 r^2 per (target, source) pair, and the reference's own r (2r - 1)
    # (m2l_aux.c:967-979), for the leaf launch and for all levels of the step
    m2l_counts = {"pairs_leaf_level": I_leaf, "pairs_all_levels": I_all,
                  "leaf_launch_gflops_2r2": 2.0 * r * r * I_leaf / (m2l_ms / 1e3) / 1e9,
                  "leaf_launch_gflops_reference_count": r * (2 * r - 1) * I_leaf / (m2l_ms / 1e3) / 1e9,
                  "stage_gflops_2r2": 2.0 * r * r * I_all / (stages["m2l"] / 1e3) / 1e9,
                  "stage_gflops_reference_count": r * (2 * r - 1) * I_all / (stages["m2l"] / 1e3) / 1e9}
    if args.mode == "mixed":
        # MMA work the leaf launch executes: every target of the level against all 189 offsets
        # (zero-filled out-of-grid sources included), per 32-component chunk hi*hi over the 256
        # outputs plus, for the first TC_SPLIT_CHUNKS chunks, the two corrections over the first
        # TC_SPLIT_ROWS outputs (the adaptive product map of the mixed mode)
        split_chunks, split_rows, chunks = 2, 64, r // 32  # TC_SPLIT_CHUNKS, TC_SPLIT_ROWS
        macs_per_pair = 32 * (split_chunks * (256 + 2 * split_rows) + (chunks - split_chunks) * 256)
        exec_flop = 2.0 * macs_per_pair * 189 * 8 ** lev
        achieved = exec_flop / (m2l_ms / 1e3) / 1e12
        # the launch is timed alone (bbfmm_b200_time_m2l, 3 launches back to back): burst peak
        roof = {"kernel": "m2l_tc2_kernel (split-bf16 tcgen05 M2L with the FP64 leading block, leaf level, "
                          "timed alone in the form the solve launches it)",
                "bound": "tensor", "achieved": achieved, "peak": bf16, "unit": "TFLOP/s", "frac": achieved / bf16,
                "peak_source": f"{peak_src} bf16 dense burst (the launch is timed alone)",
                "achieved_note": "executed BF16 MMA flops (adaptive split-BF16 product map) / launch time; "
                                 "the same launch also runs the FP64 leading block (i < 32, j < 16) on DMMA",
                "clock_normalised": {"sm_mhz_median_of_step": sm_mhz,
                                     "launch_ms_at_max_clock": m2l_ms * sm_mhz / MAX_SM_MHZ,
                                     "frac_at_max_clock": achieved * MAX_SM_MHZ / sm_mhz / bf16},
                "algorithmic_tflops": 2.0 * r * r * I_leaf / (m2l_ms / 1e3) / 1e12,
                "algorithmic_frac": 2.0 * r * r * I_leaf / (m2l_ms / 1e3) / 1e12 / bf16,
                "fp64_lead_flop": 2.0 * 32 * 16 * I_leaf,
                "traffic": TC_DRAM_BYTES_PER_CELL * 8 ** lev if TC_DRAM_BYTES_PER_CELL else None,
                "traffic_note": "ncu DRAM bytes of the level-6 launch (split rows written) scaled by cells",
                "flop_per_launch": exec_flop, "launch_ms": m2l_ms}
    else:
        flop = 2.0 * r * r * I_leaf
        achieved = flop / (m2l_ms / 1e3) / 1e12
        fp64 = args.mode == "d" and r == 256
        peak = DMMA_TFLOPS if fp64 else FP32_TFLOPS
        roof = {"kernel": "m2l_dmma_kernel (leaf level)" if fp64 else "m2l_simt_kernel (leaf level)",
                "bound": "tensor" if fp64 else "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak,
                "peak_source": "FP64 tensor (DMMA) rate, 128 flops/clock/SM at 1965 MHz" if fp64 else
                               "FP32 FMA rate, 128 lanes/SM at 1965 MHz",
                "traffic": None, "flop_per_launch": flop, "launch_ms": m2l_ms}
    # near field and passes: pairs exact from the tree, bytes of the passes
    counts = leaf_counts(x, lev)
    pairs = near_pairs(counts)
    p2p = {"pairs": pairs, "ms": stages["p2p"], "gpairs_per_s": pairs / (stages["p2p"] / 1e3) / 1e9,
           "roof_gpairs_per_s": P2P_ROOF_PAIRS / 1e9, "frac": pairs / (stages["p2p"] / 1e3) / P2P_ROOF_PAIRS,
           "roof_note": "min(FP32 issue / 7 ops per pair, MUFU rsqrt 16/clk/SM) at 1965 MHz; the mixed kernel also "
                        "does 6 FP64 operations per pair (separation and its square)"}
    pb = pass_bytes(n, lev, N, int((counts > 0).sum()), args.mode == "mixed")
    passes = {k: {"bytes": b, "ms": stages[k], "gb_per_s": b / (stages[k] / 1e3) / 1e9,
                  "frac_hbm": b / (stages[k] / 1e3) / 1e9 / hbm} for k, b in pb.items()}

    # plain FP64 GPU form of the same FMM (the speed-up denominator)
    plain = None
    if args.mode != "d" and args.plain_steps > 0:
        sol.close()
        del phi_dev
        torch.cuda.empty_cache()
        pd = Solver(n, lev, 1.0, mode="d", device=local)
        pd.set_particles(x)
        q64 = torch.as_tensor(q, device="cuda")
        ph64 = torch.empty_like(q64)
        pd.solve(q64, out=ph64)
        torch.cuda.synchronize()
        pstream = torch.cuda.ExternalStream(pd.stream)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(pstream)
        for _ in range(args.plain_steps):
            pd.solve(q64, out=ph64)
        b.record(pstream)
        torch.cuda.synchronize()
        t_plain = max_over_ranks(a.elapsed_time(b) / 1e3 / args.plain_steps)
        err_plain = rel(ph64.cpu().numpy())
        plain = {"s_per_solve": t_plain, "err_vs_direct": err_plain, "speedup": t_plain / t_dev,
                 "err_ratio": err_mode / err_plain}
        pd.close()

    # tolerance-rank mode: the SVD cut at relative singular value 1e-8 that the configuration
    # names, mixed and plain FP64 at the same truncated rank (the reference fixes r = n^3/2)
    tolr = None
    if args.mode != "d" and args.tol_rank > 0 and args.plain_steps > 0:
        res_t = {}
        for m in ("mixed", "d"):
            torch.cuda.empty_cache()
            st = Solver(n, lev, 1.0, mode=m, device=local, tol=args.tol_rank)
            st.set_particles(x)
            qt = torch.as_tensor(q, device="cuda")
            ot = torch.empty_like(qt)
            st.solve(qt, out=ot)
            reps = args.plain_steps if m == "d" else args.steps
            tt = max_over_ranks(_device_time(lambda: st.solve(qt, out=ot), reps,
                                             torch.cuda.ExternalStream(st.stream)))
            res_t[m] = {"s_per_solve": tt, "err_vs_direct": rel(ot.double().cpu().numpy()), "rank": st.rank}
            st.close()
            del qt, ot
        tolr = {"tol": args.tol_rank, "rank": res_t["d"]["rank"], "mixed": res_t["mixed"], "plain_fp64": res_t["d"],
                "speedup": res_t["d"]["s_per_solve"] / res_t["mixed"]["s_per_solve"],
                "err_ratio": res_t["mixed"]["err_vs_direct"] / res_t["d"]["err_vs_direct"]}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            Ns, ls = 65536, 5
            t_ref, cores, kind = reference_sample(Ns, ls)
            cpu = {"value": (1.0 / t_ref) * (Ns / N_FULL), "unit": "solve/s", "cores": cores, "kind": kind,
                   "sample": f"one CPU solve of N={Ns}, n=8, maxlev {ls} (2 particles/leaf, same density), "
                             f"{t_ref:.2f} s, scaled by {Ns}/{N_FULL}"}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "solve/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solve/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_dev * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": {"mixed": "bf16x3+f64", "d": "f64", "s": "f32"}[args.mode],
            "data": "synthetic (seeded uniform [0,1)^3, q~U[-1,1])",
            "config": {"workload": "bbFMM Laplace 1/r, N=4,194,304 uniform, n=8 (r=256), maxlev 7",
                       "N": N, "n": n, "maxlev": lev, "mode": args.mode,
                       "lead_fp64_components": sol.lead if args.mode == "mixed" else None,
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs and working set larger than L2 (operators 166 MB, expansions > 20 GB)"},
            "err_vs_fp64_direct": err_mode, "n_targets": N_TARGETS,
            "plain_fp64": plain,
            "tolerance_rank": tolr,
            "stages_ms": stages,
            "m2l_flops": m2l_counts,
            "p2p": p2p,
            "passes_hbm": passes,
            "setup_ms": {"host_tree": t_setup_host * 1e3, "device_tree": t_setup_dev * 1e3,
                         "note": "octree + upload of the particles, outside the metric (bitwise the same tree)"},
            "e2e": {"value": world / t_e2e, "unit": "solve/s", "h2d_bytes_per_step": N * esz,
                    "d2h_bytes_per_step": N * esz},
            "gpu_launches": launches * args.steps,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clk_now,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
