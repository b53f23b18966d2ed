#!/usr/bin/env python
"""Benchmark of the GR lattice-Boltzmann radiation step on B200.

Workload: the curved-scattering problem at scale -- Kerr-Schild M=1 a=0 on
[-6,6]^2, 400x400 cells, 64 directions, Fourier order 16, excision r <= 2.4,
RK45 tolerance 1e-10, lognormal absorption, uniform scattering, Gaussian
emission (2dradiation_b200/workloads.py: curved_scatter), synthetic seeded
fields.

A bench *step* is one time step of the solver over all 160,000 interior cells
and 64 directions (stream + moments + lambda-iteration collide, one fused
kernel).  ``value`` is cell*direction updates per second of the precision form
(FP32 intensities and stream/collide arithmetic, Kahan moments, FP64
geodesic tables) with the state resident in HBM, each step timed with CUDA
events on the library's stream and L2 flushed (256 MiB write) between timed
steps.  The plain FP64 form is measured the same way and reported beside it,
with the FP32-vs-FP64 relative error of E after the timed steps.

``e2e`` goes through the C-ABI with host buffers: every e2e step uploads the
fields and the initial intensities from pinned host memory, runs a full
2000-step simulation and reads the inertial-frame moments back.

``--impl reference`` times the reference's own CPU implementation (compiled
from its sources into oracle/_ref, else the oracle restatement) with all host
threads on the same workload, one solver step per bench step.

Run: python bench.py [--gpus N --steps K --warmup W].  N>1 runs under
torchrun as a slab decomposition (2dradiation_b200/slabs.py): the grid grows
to 400 x 400N cells, each GPU steps one 400-row band and exchanges its ghost
rows with its neighbours over NCCL before every step (weak scaling; device
time per step, max over ranks).
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

METRIC = "cell·dir updates/s, FP32+FP64-geodesic vs FP64 plain, at E rel-err ≤1e-5"
UNIT = "cell·dir updates/s"
FALLBACK_HBM_GBS = 6650.0


def args_parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=20)
    p.add_argument("--impl", default="grlbm", choices=["grlbm", "reference"])
    p.add_argument("--e2e-steps", type=int, default=2000)
    p.add_argument("--e2e-reps", type=int, default=2)
    p.add_argument("--cpu-steps", type=int, default=2, help="solver steps in the CPU-baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--nx", type=int, default=400)
    p.add_argument("--dirs", type=int, default=64)
    p.add_argument("--fourier", type=int, default=16)
    p.add_argument("--no-configs", action="store_true",
                   help="skip the flat-beam and curved-shell configurations")
    p.add_argument("--adjoint-steps", type=int, default=200,
                   help="steps of the adjoint workload (256^2 x 48, checkpoints every 20); 0 skips it")
    p.add_argument("--batch-steps", type=int, default=64,
                   help="timed steps of the batched form (64 uneven problems); 0 skips it")
    p.add_argument("--profile", default=None,
                   choices=["fp32", "fp64", "fast64", "fp32-adaptive", "fp64-adaptive", "batch", "adjoint"],
                   help="instead of measuring: build one problem and run --profile-steps steps of it, one call "
                        "per step, for a profiler to capture (no timing, no JSON line)")
    p.add_argument("--profile-steps", type=int, default=6)
    p.add_argument("--profile-workload", default="curved_scatter")
    p.add_argument("--profile-batch", type=int, default=16, help="problems of the batched form in --profile batch")
    return p.parse_args()


def workload_name(a) -> str:
    return (f"curved_scatter {a.nx}x{a.nx} cells x {a.dirs} directions, Fourier order {a.fourier}, "
            "Kerr-Schild M=1 a=0 on [-6,6]^2, excision r<=2.4, RK45 tol 1e-10")


def dist_setup(a):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1 and a.impl == "grlbm":
        import torch.distributed as dist
        from datetime import timedelta
        import torch
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(x: float, pg, device=None) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, device=None):
    if pg is not None:
        import torch
        t = torch.zeros(1, device=device)
        pg.all_reduce(t)


class Clocks:
    """nvidia-smi sampler for the SM clock and throttle reasons while the GPU works."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}

        def num(s):
            try:
                return float(s)
            except ValueError:
                return None
        sm = [num(r[1]) for r in self.rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in self.rows if num(r[2]) is not None]
        pw = [num(r[3]) for r in self.rows if num(r[3]) is not None]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        loaded = [s for s, p in zip(sm, pw) if p is not None and p > 300] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows), "power_w_max": max(pw) if pw else None}


def hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            v = json.loads(p.read_text()).get("hbm_gbs")
            if v:
                return float(v), "measured"
        except (ValueError, OSError):
            pass
    return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(kernel: str, key: str = "dram_bytes_per_launch"):
    """DRAM bytes per launch of `kernel` (or another per-launch figure, `key`)
    from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        return d.get(kernel, {}).get(key)
    except (ValueError, OSError):
        return None


# FP64 peak of a B200: 148 SMs x 64 FP64 FMA lanes x 2 FLOP x 1.965 GHz
FP64_PEAK_TFLOPS_NOMINAL = 148 * 64 * 2 * 1.965e9 / 1e12


def table_build_line(fp32):
    """The geodesic table build of the bench workload: its time, its RK45
    trials, and its FP64 rate over the whole build from the FP64 operations
    ncu counted in k_geodesic at this workload (DADD + DMUL + 2 DFMA)."""
    flop = profiled_traffic("k_geodesic", "fp64_flop_per_launch")
    ms = fp32["table_ms"]
    out = {"ms": ms, "rk_substeps": fp32["rk_substeps"], "fp64_flop": flop,
           "achieved_fp64_tflops": flop / (ms * 1e-3) / 1e12 if flop and ms > 0 else None,
           "fp64_peak_tflops_nominal": FP64_PEAK_TFLOPS_NOMINAL,
           "note": "k_geodesic + k_fourier_project + k_departure, CUDA events; FP64 operations from the committed "
                   "ncu count of k_geodesic (built without contraction, as the reference rounds)"}
    if out["achieved_fp64_tflops"]:
        out["fp64_frac_nominal"] = out["achieved_fp64_tflops"] / FP64_PEAK_TFLOPS_NOMINAL
    return out


def time_steps(G, r, steps: int, warmup: int, flush, advance):
    """Per-step device time (ms) on the library's stream, L2 flushed between
    steps; `advance` enqueues one step (with its ghost-row exchange on
    several GPUs)."""
    import torch
    ext = torch.cuda.ExternalStream(r.stream)
    with torch.cuda.stream(ext):
        for _ in range(warmup):
            advance()
            flush.zero_()
        ext.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for s, e in ev:
            s.record(ext)
            advance()
            e.record(ext)
            flush.zero_()
        ext.synchronize()
    return [s.elapsed_time(e) for s, e in ev]


def open_form(G, case, prec, world, rank, local, pg):
    """A context for one form: the whole grid on one GPU, or this rank's band
    of a slab decomposition (ghost rows exchanged before every step)."""
    if world == 1:
        r = G.prepare(case, prec, device=local)
        return r, (lambda: r.step_async(1)), None
    S = importlib.import_module("2dradiation_b200.slabs")
    r, slab = S.open_slab(case, prec, rank, world, local, pg)
    return r, (lambda: slab.step(1)), slab


def run_configs(G, W, local):
    """The two smaller configurations at their full sizes -- the flat beam
    (100^2 x 20, 500 steps) and the curved shell (200^2 x 32, 1000 steps) --
    in the three forms, and the bench workload with adaptive streaming (50
    steps) in the plain and precision forms, with each form's relative error
    of E against the plain form.  Device time of the whole run
    with CUDA events (graph-replayed steps, inputs resident, no L2 flush
    between steps)."""
    import torch
    out = {}
    for name, case, forms in (
            ("flat_beam 100x100 x 20 directions, 500 steps", W.flat_beam(),
             (G.PLAIN_FP64, G.PRECISION_FP32, G.FAST_FP64)),
            ("curved_shell 200x200 x 32 directions, Fourier order 5, 1000 steps", W.curved_shell(),
             (G.PLAIN_FP64, G.PRECISION_FP32, G.FAST_FP64)),
            ("curved_scatter adaptive (CurvedAdaptive) 400x400 x 64 directions, Fourier order 16, 50 steps",
             dict(W.curved_scatter(steps=50), streaming_type=W.CURVED_ADAPTIVE), (G.PLAIN_FP64, G.PRECISION_FP32))):
        n = int(case["n_steps"])
        units = int(case["nx_"]) * int(case["ny_"]) * int(case["n_dir"]) * n
        res, E = {}, {}
        for prec in forms:
            with G.prepare(case, prec, device=local) as r:
                ext = torch.cuda.ExternalStream(r.stream)
                with torch.cuda.stream(ext):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(ext)
                    r.step_async(n)
                    e1.record(ext)
                    ext.synchronize()
                key = {G.PLAIN_FP64: "fp64", G.PRECISION_FP32: "fp32", G.FAST_FP64: "fast64"}[prec]
                res[key] = units / (e0.elapsed_time(e1) / 1e3)
                E[key] = r.moments_if()["E"]
        entry = {"cell_dir_per_s": res}
        if "fp32" in E:
            entry["E_rel_l2_fp32_vs_fp64"] = float(np.linalg.norm(E["fp32"] - E["fp64"]) / np.linalg.norm(E["fp64"]))
        if "fast64" in E:
            entry["E_rel_l2_fast64_vs_fp64"] = float(np.linalg.norm(E["fast64"] - E["fp64"]) / np.linalg.norm(E["fp64"]))
        out[name] = entry
    return out


def run_batched(G, W, a, local, world=1, rank=0, pg=None, dev=None):
    """The batched form on 64 uneven problems (grid 64^2..512^2, 16..64
    directions, flat or Schwarzschild, seed 10): after autotuning the launch
    shape, `batch_steps` steps of all problems through the batch, against the
    same problems stepped through their own contexts (one stream each,
    enqueued back to back).  Both are timed after an untimed round of the same
    length, which captures their 32-step graphs.  On N GPUs the problems are
    dealt to the ranks as independent replicas (share_problems: balanced by
    estimated cost, no communication); each rank batches its own, and a
    timed region ends with the slowest rank."""
    import torch
    allc = W.batch_instances(count=64, seed=10, steps=a.batch_steps)
    units = sum(int(c["nx_"]) * int(c["ny_"]) * int(c["n_dir"]) for c in allc)
    deal = G.share_problems(allc, world)
    cases = [allc[k] for k in deal[rank]]
    probs = [G.prepare(c, G.PRECISION_FP32, device=local) for c in cases]

    def start():
        torch.cuda.synchronize()
        barrier(pg, dev)
        torch.cuda.synchronize()
        return time.perf_counter()

    try:
        for r in probs:  # an untimed round: graphs captured, caches warm
            r.step(a.batch_steps)
        t0 = start()
        for r in probs:
            r.step_async(a.batch_steps)
        for r in probs:
            r.sync()
        single_s = max_over_ranks(time.perf_counter() - t0, pg, dev)
        b = G.Batch(probs) if probs else None  # a rank may be dealt no problem
        try:
            choice = b.autotune(3) if b else None
            if b:
                b.step(a.batch_steps)
            t0 = start()
            if b:
                b.step(a.batch_steps)
            batch_s = max_over_ranks(time.perf_counter() - t0, pg, dev)
        finally:
            if b:
                b.close()
    finally:
        for r in probs:
            r.close()
    return {"problems": len(allc), "cell_dir_per_step": units, "steps": a.batch_steps,
            "value": units * a.batch_steps / batch_s, "unit": UNIT,
            "separate_contexts": units * a.batch_steps / single_s, "autotune": choice,
            "replicas": world, "problems_per_gpu": [len(x) for x in deal],
            "timing": "host clock around the synchronous batch step, the slowest rank's (the autotuned launch "
                      "shape, rank 0's: blocks_per_sm 0 = the problems' own kernels launched concurrently, -m = the "
                      "same on cost-weighted shares of m GPUs' worth of resident blocks, >= 1 = one persistent "
                      "launch per step; 32-step graphs), after an untimed round"}


def run_adjoint(G, W, a, local):
    """The adjoint workload (Schwarzschild 256^2 x 48 directions, Gaussian-sum
    eta and kappaA, `adjoint_steps` steps, checkpoints every 20): the plain
    forward alone, the checkpointed forward (after an untimed one that
    allocates the checkpoints), and the backward (recompute + adjoint), each
    timed on the host around synchronous calls; the inverse-table time
    includes the adjoint's set-up allocations."""
    import torch
    case = W.adjoint_case(steps=a.adjoint_steps)
    target = W.adjoint_case(steps=a.adjoint_steps, seeds=(7, 8))
    n = a.adjoint_steps
    with G.prepare(target, G.PLAIN_FP64, device=local) as t:
        t.step(n)
        Et = t.moments_if()["E"]
    r = G.prepare(case, G.PLAIN_FP64, device=local)
    try:
        I0 = np.zeros(r.nxy * r.nd)
        t0 = time.perf_counter()
        adj = G.Adjoint(r, 20)
        table_s = time.perf_counter() - t0
        r.set_intensity(I0)
        r.step(n)
        r.set_intensity(I0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r.step(n)
        plain_s = time.perf_counter() - t0
        r.set_intensity(I0)
        adj.forward(n)  # untimed: the first forward allocates the checkpoints
        r.set_intensity(I0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        adj.forward(n)
        fwd_s = time.perf_counter() - t0
        E = r.moments_if()["E"]
        nx = r.nx
        mask = np.zeros((r.ny, nx), bool)
        mask[1:-1, 1:-1] = True
        dLdE = np.where(mask.ravel(), E - Et, 0.0)
        t0 = time.perf_counter()
        g = adj.backward(dLdE)
        bwd_s = time.perf_counter() - t0
        adj.close()
    finally:
        r.close()
    return {"workload": "adjoint: Schwarzschild 256x256 x 48 directions, eta/kappaA sums of 8 Gaussians, "
                        f"{n} steps, checkpoints every 20, loss 0.5|E - E*|^2",
            "loss": 0.5 * float(np.sum(dLdE ** 2)),
            "inverse_table_s": table_s, "plain_forward_ms_per_step": 1e3 * plain_s / n,
            "checkpointed_forward_ms_per_step": 1e3 * fwd_s / n,
            "backward_ms_per_step": 1e3 * bwd_s / n,
            "adjoint_step_over_forward_step": bwd_s / plain_s,
            "grad_norms": {k: float(np.linalg.norm(v)) for k, v in g.items()},
            "timing": "host clock around synchronous calls; the backward includes the forward recompute"}


def run_profile(a):
    """A problem for a profiler to capture: the bench workload (or
    --profile-workload) in one form, stepped one call at a time, so that
    the profiler can skip the warm-up launches; or the batched form
    (--profile-batch uneven problems of seed 10); or the adjoint workload
    (forward and one backward of --profile-steps steps)."""
    G = importlib.import_module("2dradiation_b200")
    W = G.workloads
    n = a.profile_steps
    if a.profile == "batch":
        probs = [G.prepare(c, G.PRECISION_FP32) for c in W.batch_instances(count=a.profile_batch, seed=10)]
        with G.Batch(probs) as b:
            # the persistent kernel at the most resident blocks per SM it allows
            for bps in (4, 3, 2, 1):
                try:
                    b.set_shape(bps, True)
                    break
                except G.GrlbmError:
                    continue
            for _ in range(n):
                b.step(1)
        print("profile: batch of", a.profile_batch, "E sum", float(sum(r.moments_if()["E"].sum() for r in probs)))
        for r in probs:
            r.close()
        return
    if a.profile == "adjoint":
        r = G.prepare(W.adjoint_case(steps=n), G.PLAIN_FP64)
        with G.Adjoint(r, 20) as adj:
            r.set_intensity(np.zeros(r.nxy * r.nd))
            adj.forward(n)
            g = adj.backward(r.moments_if()["E"])
        print("profile: adjoint", n, "steps, |dL/deta|", float(np.linalg.norm(g["eta"])))
        r.close()
        return
    kw = dict(nx_=a.nx, ny_=a.nx, n_dir=a.dirs, steps=n)
    if a.profile_workload != "flat_beam":
        kw["n_fourier"] = a.fourier
    case = W.make_case(a.profile_workload, **kw)
    if a.profile.endswith("adaptive"):
        case["streaming_type"] = W.FLAT_ADAPTIVE if case["streaming_type"] == W.FLAT_FIXED else W.CURVED_ADAPTIVE
    prec = G.PRECISION_FP32 if a.profile.startswith("fp32") else (G.FAST_FP64 if a.profile == "fast64" else G.PLAIN_FP64)
    with G.prepare(case, prec) as r:
        for _ in range(n):
            r.step(1)
        print("profile:", a.profile, a.profile_workload, a.nx, a.dirs, "E sum", float(r.moments_if()["E"].sum()))


def run_e2e(G, W, case, prec, a, world, rank, local, pg, dev):
    """End to end through the C-ABI with pinned host buffers: every rep
    uploads the fields and the initial intensities, runs the whole
    `e2e_steps`-step simulation and reads the moments back (host clock, max
    over ranks, median of the timed reps after an untimed one).  Returns the
    seconds per rep and the moments of the last rep."""
    import torch
    f = case["fields"]
    host = {k: torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64)).pin_memory().numpy()
            for k, v in f.items() if k != "is_initial"}
    I0 = torch.zeros(W.nxy(case) * a.dirs, dtype=torch.float64).pin_memory().numpy()
    mom = {k: torch.zeros(W.nxy(case), dtype=torch.float64).pin_memory().numpy()
           for k in ("E", "Fx", "Fy", "Pxx", "Pxy", "Pyy")}
    r, advance, slab = open_form(G, case, prec, world, rank, local, pg)
    e2e_t = []
    try:
        for rep in range(a.e2e_reps + 1):
            barrier(pg, dev)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r.set_fields(host)
            r.set_intensity(I0)
            if slab is None:
                r.step(a.e2e_steps)
            else:
                slab.step(a.e2e_steps)
            r.moments_if(mom)
            t1 = time.perf_counter()
            if rep > 0:
                e2e_t.append(t1 - t0)
        lo, hi = slab.band if slab is not None else (1, a.nx + 1)
        band = {k: v[lo * (a.nx + 2):hi * (a.nx + 2)].copy() for k, v in mom.items()}
        iters = r.stats()["average_iterations"]
    finally:
        r.close()
    return max_over_ranks(statistics.median(e2e_t), pg, dev), band, iters


def run_grlbm(a, world, rank, local, pg):
    import torch
    G = importlib.import_module("2dradiation_b200")
    W = G.workloads
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # one 400-row band per GPU: the grid grows with the GPU count (weak scaling)
    case = W.curved_scatter(nx_=a.nx, ny_=a.nx * world, n_dir=a.dirs, n_fourier=a.fourier, steps=a.e2e_steps)
    ncell, nd = a.nx * a.nx, a.dirs
    units = ncell * nd
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    peak, peak_kind = hbm_peak()
    out = {}
    with Clocks(local) as clk:
        forms = {}
        states = {}
        for name, prec in (("fp32", G.PRECISION_FP32), ("fp64", G.PLAIN_FP64), ("fast64", G.FAST_FP64)):
            r, advance, slab = open_form(G, case, prec, world, rank, local, pg)
            st = r.stats()
            barrier(pg, dev)
            ms = time_steps(G, r, a.steps, a.warmup, flush, advance)
            total = max_over_ranks(sum(ms), pg, dev)
            forms[name] = {"ms": ms, "total_ms": total, "table_ms": st["table_ms"], "rk_substeps": st["rk_substeps"]}
            lo, hi = slab.band if slab is not None else (1, a.nx + 1)
            states[name] = {k: v[lo * (a.nx + 2):hi * (a.nx + 2)] for k, v in r.moments_if().items()}
            forms[name]["iters"] = r.stats()
            r.close()
        # e2e through the C-ABI with pinned host buffers, both forms; their
        # moments after the whole run give the metric's accuracy condition
        e2e = {}
        if a.e2e_reps > 0:
            for name, prec in (("fp32", G.PRECISION_FP32), ("fp64", G.PLAIN_FP64), ("fast64", G.FAST_FP64)):
                e2e[name] = run_e2e(G, W, case, prec, a, world, rank, local, pg, dev)
        batched = run_batched(G, W, a, local, world, rank, pg, dev) if a.batch_steps > 0 else None
        other = run_configs(G, W, local) if not a.no_configs and world == 1 else None
        adjoint = run_adjoint(G, W, a, local) if a.adjoint_steps > 0 and world == 1 else None
    clocks = clk.summary()

    fp32, fp64, fast = forms["fp32"], forms["fp64"], forms["fast64"]
    value = world * units * a.steps / (fp32["total_ms"] / 1e3)
    plain = world * units * a.steps / (fp64["total_ms"] / 1e3)
    fast_value = world * units * a.steps / (fast["total_ms"] / 1e3)
    # algorithmic bytes per cell*direction: I read + written, 4 inputs and 6
    # moments per cell shared by the directions
    b32 = 2 * 4 + (4 + 6) * 4 / nd
    b64 = 2 * 8 + (4 + 6) * 8 / nd
    avg32 = statistics.mean(fp32["ms"]) / 1e3
    avg64 = statistics.mean(fp64["ms"]) / 1e3
    avgf = statistics.mean(fast["ms"]) / 1e3
    ach32 = b32 * units / avg32 / 1e9
    ach64 = b64 * units / avg64 / 1e9
    achf = b64 * units / avgf / 1e9
    rel = lambda x, y: float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
    if "fp32" in e2e and "fp64" in e2e:
        m32, m64 = e2e["fp32"][1], e2e["fp64"][1]
        accuracy = {k + "_rel_l2_fp32_vs_fp64": max_over_ranks(rel(m32[k], m64[k]), pg, dev)
                    for k in ("E", "Fx", "Fy")}
        accuracy.update({"after_steps": a.e2e_steps, "from": "the e2e runs of both forms (same initial state)",
                         "lambda_iterations_avg": {"fp32": e2e["fp32"][2], "fp64": e2e["fp64"][2]}})
    else:
        accuracy = {k + "_rel_l2_fp32_vs_fp64": rel(states["fp32"][k], states["fp64"][k]) for k in ("E", "Fx", "Fy")}
        accuracy["after_steps"] = a.warmup + a.steps
    # the fast FP64 form against the plain form (bit-identical to the oracle
    # at this size) on the same runs
    if "fast64" in e2e and "fp64" in e2e:
        mf, m64 = e2e["fast64"][1], e2e["fp64"][1]
        fast_accuracy = {k + "_rel_l2_fast64_vs_fp64": max_over_ranks(rel(mf[k], m64[k]), pg, dev)
                         for k in ("E", "Fx", "Fy")}
        fast_accuracy.update({"after_steps": a.e2e_steps, "lambda_iterations_avg": e2e["fast64"][2]})
    else:
        fast_accuracy = {k + "_rel_l2_fast64_vs_fp64": rel(states["fast64"][k], states["fp64"][k])
                         for k in ("E", "Fx", "Fy")}
        fast_accuracy["after_steps"] = a.warmup + a.steps

    def e2e_line(name):
        if name not in e2e:
            return None
        sec = e2e[name][0]
        return {"value": world * units * a.e2e_steps / sec, "unit": UNIT,
                "h2d_bytes_per_step": int(8 * (6 * W.nxy(case) + W.nxy(case) * nd)),
                "d2h_bytes_per_step": int(8 * 6 * W.nxy(case)),
                "step": f"C-ABI: set fields + set intensities (host) + {a.e2e_steps} solver steps + moments to host",
                "seconds_per_step": sec}
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": fp32["total_ms"] / a.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": workload_name(a),
            "form": "precision: FP32 intensities and stream/collide, Kahan FP32 moments, FP64 geodesic tables",
            "step": "one time step (fused stream + moments + lambda-iteration collide) over all interior cells",
            "l2": "flushed between timed steps by a 256 MiB write (untimed)",
            "parallelism": "single GPU" if world == 1 else
            f"slab decomposition: {world} bands of {a.nx} rows, one per GPU, ghost rows exchanged over NCCL every step",
            "global_batch": units,
        },
        "roofline": {
            "bound": "hbm",
            "achieved": ach32,
            "peak": peak,
            "peak_kind": peak_kind,
            "unit": "GB/s",
            "frac": ach32 / peak,
            "traffic": profiled_traffic("k_step_prec"),
            "algorithmic_bytes_per_update": b32,
            "kernel": "k_step_prec<curved>",
        },
        "plain_fp64": {
            "value": plain,
            "ms_per_step": fp64["total_ms"] / a.steps,
            "roofline_frac": ach64 / peak,
            "achieved_gbs": ach64,
            "algorithmic_bytes_per_update": b64,
            "traffic": profiled_traffic("plain_step"),
            "kernels": "k_stream_plain + k_collide_plain (fixed streaming; traffic per step, both kernels)",
        },
        "fast_fp64": {
            "value": fast_value,
            "ms_per_step": fast["total_ms"] / a.steps,
            "roofline_frac": achf / peak,
            "achieved_gbs": achf,
            "algorithmic_bytes_per_update": b64,
            "traffic": profiled_traffic("k_step_fast64"),
            "kernel": "k_step_fast64<curved> (FP64, contracted FMAs, 32-byte packed records; matches the "
                      "reference to 1e-12 where the lambda iteration's cycle count is not set by rounding noise)",
            "accuracy": fast_accuracy,
            "e2e": e2e_line("fast64"),
            "fast_vs_plain": fast_value / plain,
        },
        "precision_vs_plain": value / plain,
        # as if the step time scaled with the lambda iterations each form ran
        # (the FP32 form's moment-space iterations cost O(1) per cell, so this
        # bounds the iterations' share of the ratio from above)
        "precision_vs_plain_iteration_normalised": value / plain * fp32["iters"]["average_iterations"]
        / max(fp64["iters"]["average_iterations"], 1e-30),
        "accuracy": accuracy,
        "table_build_ms": {"fp32": fp32["table_ms"], "fp64": fp64["table_ms"], "fast64": fast["table_ms"]},
        "table_build": table_build_line(fp32),
        "lambda_iterations": {"fp32_avg": fp32["iters"]["average_iterations"],
                              "fp64_avg": fp64["iters"]["average_iterations"],
                              "fast64_avg": fast["iters"]["average_iterations"],
                              "max": fp64["iters"]["max_iterations"]},
        "e2e": e2e_line("fp32"),
        "plain_fp64_e2e": e2e_line("fp64"),
        "gpu_launches": a.steps,
        "batched": batched,
        "other_configs": other,
        "adjoint": adjoint,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(a)
    return line


def cpu_run(a, steps: int):
    import oracle
    W = importlib.import_module("2dradiation_b200.workloads")
    case = W.curved_scatter(nx_=a.nx, ny_=a.nx, n_dir=a.dirs, n_fourier=a.fourier, steps=steps)
    kind = "ref_fast" if oracle.available("ref_fast") else "oracle"
    cores = os.cpu_count() or 1
    res = oracle.run(case, kind, n_threads=cores)
    return res, kind, cores


def cpu_baseline(a):
    res, kind, cores = cpu_run(a, a.cpu_steps)
    units = a.nx * a.nx * a.dirs * a.cpu_steps
    return {"value": units / res["computation_time_s"], "unit": UNIT, "cores": cores,
            "kind": "reference" if kind == "ref_fast" else "port",
            "sample": f"{a.cpu_steps} solver steps of the same workload after its geodesic table build "
                      f"({res['table_time_s']:.1f} s, untimed); reference built with -O3 -ffast-math -fopenmp",
            "table_build_s": res["table_time_s"]}


def run_reference(a, world, rank):
    """The reference's CPU path on the bench's own grid, one solver step per
    bench step.  When the requested steps would not finish in about two and a
    half minutes, fewer steps are timed (the rate is per cell*direction
    update, and every step does the same work): the sample says how many."""
    if rank != 0:
        return None
    cores = os.cpu_count() or 1
    rate_guess = 1.2e6 * cores  # measured: 1.9e7 cell*dir/s on 16 host cores at 400x400x64
    per_step = a.nx * a.nx * a.dirs / rate_guess
    budget = max(2, int(150.0 / per_step))
    warm = min(a.warmup, max(1, budget // 10))
    timed = max(1, min(a.steps, budget - warm))
    res, kind, cores = cpu_run(a, warm + timed)
    t = res["step_times"][warm:warm + timed]
    units = a.nx * a.nx * a.dirs
    value = units * timed / float(np.sum(t))
    sample = (f"{timed} timed solver steps (of {a.steps} requested) after {warm} warm-up steps on the full "
              f"{a.nx}x{a.nx} grid, {a.dirs} directions, Fourier order {a.fourier}; geodesic table build "
              f"{res['table_time_s']:.1f} s untimed; "
              f"{'reference built -O3 -ffast-math -fopenmp' if kind == 'ref_fast' else 'oracle restatement'}")
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * float(np.mean(t)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": workload_name(a), "step": "one solver time step on the host cores (OpenMP)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores,
                         "kind": "reference" if kind == "ref_fast" else "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    a = args_parse()
    if a.profile:
        run_profile(a)
        return
    world, rank, local, pg = dist_setup(a)
    try:
        if a.impl == "reference":
            line = run_reference(a, world, rank)
        else:
            line = run_grlbm(a, world, rank, local, pg)
        if rank == 0 and line is not None:
            print(json.dumps(line))
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
