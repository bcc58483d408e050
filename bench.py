#!/usr/bin/env python
"""Benchmark of the fluid-solid RK4 time step (Gcell-updates/s, % of HBM roofline).

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

One "step" is one RK4 time step of the whole model (four fused stage launches
plus the interface filter / receiver launch). The default workload is the
4096 x 2048 curvilinear model (sinusoidal seafloor on the middle row, +-5%
correlated perturbations, 20-cell CFS-PML), seeded and synthetic; its state
and coefficients (~0.7 GB) exceed the 126 MB L2, so no flush is needed.

value  = cells x steps / device time (CUDA events on the solver's stream, max
         over ranks), cells = nx (nz_f + nz_s) as the reference counts them.
e2e    = the same metric through the public API with host buffers: model
         upload from pinned host memory, the steps, and the receiver read-back
         (after one untimed upload), with the three parts' times.
roofline: algorithmic bytes per step (16 S + 4 M floats per cell: 464 B solid,
         288 B fluid, +256 B per PML strip cell and direction) over the summed
         average durations of the four stage launches.
With N > 1 every rank runs its own copy of the workload (independent shots):
weak scaling, no data-path collective.
other_workloads.reference_cuda_build: the reference's own CUDA build
         (oracle/_ref/main_debug, compiled from its sources) and this library's
         drop-in CLI on the same JSON models, per-step time from the difference
         of the fastest wall times of a short and a long run (start-up and
         model loading cancel), snapshots off.
fp64_error: relative L2 distance of every result to the FP64 oracle over a
         bounded number of steps (the largest over the state fields).
"""
from __future__ import annotations

import argparse
import importlib
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
modelgen = importlib.import_module("marineseis-fdm-2d_b200.modelgen")

WORKLOADS = {
    "curvilinear_4096x2048": lambda: modelgen.curvilinear_4096x2048(nt=10),
    "curvilinear_2048x1024": lambda: modelgen.curvilinear(2048, 1024, zeta0=511, nt=10),
    "curvilinear_1200x800": lambda: modelgen.curvilinear_1200x800(nt=10),
    "flat_400x400": lambda: modelgen.flat_400x400(nt=10),
}
DEFAULT_WORKLOAD = "curvilinear_4096x2048"
METRIC = "Gcell-updates/s (fluid-solid RK4 step, % HBM roofline)"


def bench_config(args, model, world: int) -> dict:
    """The `config` object both arms print (the same workload)."""
    return {"workload": args.workload, "nx": model.nx, "nz_f": model.nz_f,
            "nz_s": model.nz_s, "cells": model.cells, "npd": model.npd,
            "parallelism": f"independent shots x{world}",
            "l2": "inputs larger than L2 (state + coefficients > 126 MB)"}


def rel_l2(a, b) -> float:
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / n) if n > 0 else float(np.linalg.norm(a))


STATE = ("fluid_vx", "fluid_vz", "fluid_p", "solid_vx", "solid_vz", "solid_sx", "solid_sz",
         "solid_sxz")


def fp64_error(mfdm, model, steps: int, device: int, shot=None) -> dict:
    """Largest relative L2 distance over the eight state fields between the CUDA
    path and the FP64 oracle after `steps` steps from rest (a bounded sample of
    the workload; the oracle runs on the host). `shot` = (x, z, fpeak, beta0)
    sets the source and frequency of a batched shot."""
    import copy
    from oracle import pyoracle
    pyoracle.build()
    m = copy.deepcopy(model)
    if shot is not None:
        m.src_x, m.src_z, m.fpeak, m.beta0 = [shot[0]], [shot[1]], shot[2], shot[3]
    with mfdm.Solver.from_model(m, device=device) as s:
        s.set_shot(0, reset=True)
        s.step(steps)
        ours = {n: s.field(n) for n in STATE}
    ref = pyoracle.forward(m, steps, pyoracle.record_gap(m.dt), 64, final_fields=True)
    refs = dict(zip(STATE, list(ref["fluid"]) + list(ref["solid"])))
    errs = {n: rel_l2(ours[n], refs[n]) for n in STATE}
    worst = max(errs, key=errs.get)
    return {"rel_l2": float(f"{errs[worst]:.3e}"), "field": worst, "steps": steps}


def wall_run(binary: str, jpath: str, out: str) -> float:
    t0 = time.perf_counter()
    subprocess.run([binary, jpath, out], check=True, stdout=subprocess.DEVNULL,
                   stderr=subprocess.DEVNULL)
    return time.perf_counter() - t0


def reference_cuda_build(workloads, repeats: int = 3) -> dict:
    """The reference's CUDA build (oracle/_ref/main_debug, its own sources compiled
    for sm_100a) and this library's drop-in CLI on the same JSON models, snapshots
    off (snapshot > nt). Per-step time = (wall time of the long run - that of the
    short run) / step difference, each the fastest of `repeats` interleaved runs
    (src/main.cu:136-213 is the reference's timed loop; start-up and model reading
    cancel in the difference). Each arm's long run is sized to a few seconds of
    stepping, so the faster library takes more steps than the reference:
    workloads are (name, build(nt), (n1, n2) of the reference, (n1, n2) of the
    library)."""
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "main_debug")
    our_bin = os.path.join(ROOT, "marineseis-fdm-2d_b200", "bin", "main_debug")
    if not (os.path.exists(ref_bin) and os.path.exists(our_bin)):
        return {"unavailable": "oracle/_ref/main_debug not built (needs the reference sources)"}
    out = {}
    for name, build, ref_steps, our_steps in workloads:
        work = tempfile.mkdtemp(prefix="mfdm_refbuild_")
        try:
            row = {}
            for label, binary, (n1, n2) in (("reference", ref_bin, ref_steps),
                                            ("library", our_bin, our_steps)):
                model = build(n1)
                model.snapshot = n2 + 1
                j1 = modelgen.write_model(model, work, name=f"{label}_short")
                cfg = json.load(open(j1))
                cfg["base"]["nt"] = n2
                j2 = os.path.join(work, f"{label}_long.json")
                with open(j2, "w") as f:
                    json.dump(cfg, f)
                wall_run(binary, j1, os.path.join(work, "out"))  # page the model files in
                runs = {n1: [], n2: []}
                for _ in range(repeats):
                    for nt, j in ((n1, j1), (n2, j2)):
                        runs[nt].append(wall_run(binary, j, os.path.join(work, "out")))
                ms = (min(runs[n2]) - min(runs[n1])) / (n2 - n1) * 1e3
                row[label] = {"ms_per_step": round(ms, 4),
                              "gcells": round(model.cells / (ms / 1e3) / 1e9, 3), "steps": [n1, n2]}
            row["speedup"] = round(row["reference"]["ms_per_step"] / row["library"]["ms_per_step"], 2)
            out[name] = row
        finally:
            shutil.rmtree(work, ignore_errors=True)
    return out


def algorithmic_bytes(m) -> int:
    """Bytes per step a classical-RK4 sweep must move (16 S + 4 M floats per cell)."""
    fluid = m.nx * m.nz_f * (16 * 3 + 4 * 6) * 4
    solid = m.nx * m.nz_s * (16 * 5 + 4 * 9) * 4
    strips = 2 * m.npd * (m.nz_f - 3) + 2 * m.npd * (m.nz_s - 3) + m.npd * (m.nx - 6)
    return fluid + solid + strips * 16 * 4 * 4


def batched_bytes(m, nshots: int) -> int:
    """Bytes per step of `nshots` shots of one model when the coefficients are
    read once for all shots (each shot still moves its own 16 state floats per
    field and cell and its ADE memory)."""
    state = m.nx * m.nz_f * 16 * 3 + m.nx * m.nz_s * 16 * 5
    strips = 2 * m.npd * (m.nz_f - 3) + 2 * m.npd * (m.nz_s - 3) + m.npd * (m.nx - 6)
    coef = m.nx * m.nz_f * 4 * 6 + m.nx * m.nz_s * 4 * 9
    return (nshots * (state + strips * 16 * 4) + coef) * 4


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.device), "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.25)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_oracle_rate(model, target_s: float, max_steps: int):
    """Times the oracle (FP32 CPU restatement, all host threads) on a bounded sample."""
    from oracle import pyoracle
    pyoracle.build()
    st = pyoracle.Stepper(model, 32)
    threads = pyoracle.max_threads()
    st.step(1)  # warm-up (first touch, thread pool)
    done, t0 = 0, time.perf_counter()
    while done < max_steps and (time.perf_counter() - t0) < target_s:
        st.step(1)
        done += 1
    secs = time.perf_counter() - t0
    st.close()
    return model.cells * done / secs / 1e9, threads, done, secs


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as td
        from datetime import timedelta
        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = td
    return world, rank, local, dist


def max_over_ranks(dist, value: float, local: int) -> float:
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, local: int):
    if dist is not None:
        dist.barrier(device_ids=[local])


def run_reference(args, model, world, rank):
    """Reference arm: the reference has no CPU implementation of this path, so the
    CPU restatement in oracle/ (its operation order, FP32) is timed on the host."""
    if rank != 0:
        return
    budget = 150.0  # seconds of CPU work for warm-up + timed steps together
    from oracle import pyoracle
    pyoracle.build()
    st = pyoracle.Stepper(model, 32)
    threads = pyoracle.max_threads()
    t0 = time.perf_counter()
    st.step(1)
    per_step = time.perf_counter() - t0
    warm = max(0, min(args.warmup - 1, int(budget * 0.1 / max(per_step, 1e-6))))
    st.step(warm)
    steps = max(1, min(args.steps, int(budget * 0.9 / max(per_step, 1e-6))))
    t0 = time.perf_counter()
    st.step(steps)
    secs = time.perf_counter() - t0
    st.close()
    value = model.cells * steps / secs / 1e9
    sample = (f"{steps} of {args.steps} requested steps of {args.workload} "
              f"({model.cells} cells) after {warm + 1} warm-up steps")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "Gcell/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": warm + 1,
        "ms_per_step": round(secs / steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(args, model, world),
        "cpu_baseline": {"value": round(value, 4), "unit": "Gcell/s", "cores": threads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 4), "unit": "Gcell/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def batched_shots(model, n: int, seed: int = 2):
    """n shots spread along the source row, Ricker f in U[10, 25] Hz (seeded),
    PML beta0 by the generators' rule for that frequency."""
    rng = np.random.default_rng(seed)
    lo, hi = model.npd + 10, model.nx - model.npd - 10
    xs = np.linspace(lo, hi, n).round().astype(int)
    fs = rng.uniform(10.0, 25.0, n)
    z = int(model.src_z[0])
    return [(int(x), z, float(f), float(modelgen.beta0_rule(model, f))) for x, f in zip(xs, fs)]


def batched_rate(mfdm, model, device: int, warmup: int, nshots: int = 64, steps: int = 300):
    """Shot-steps/s of one batch (one launch per RK stage for all shots) against
    the same shots run one after another through single-shot handles, device
    time (CUDA events) over `steps` steps each. Both arms pick their segment
    height with the autotuner first."""
    import copy
    shots = batched_shots(model, nshots)
    with mfdm.Batch.from_model(model, shots, device=device) as b:
        tile_b = b.autotune()
        b.step(warmup)
        tb, _ = b.time_steps(steps)
    loop_ms = 0.0
    m1 = copy.deepcopy(model)
    with mfdm.Solver.from_model(m1, device=device) as s1:
        tile_1 = s1.autotune()
        for x, z, f, be in shots:
            m1.src_x, m1.src_z, m1.fpeak, m1.beta0 = [x], [z], f, be
            s1.load_model(m1)
            s1.set_shot(0, reset=True)
            s1.step(warmup)
            t1, _ = s1.time_steps(steps)
            loop_ms += t1
    cells = model.cells * nshots * steps
    peak, _ = peaks()
    shared = batched_bytes(model, nshots) * steps / (tb / 1e3) / 1e9
    unshared = algorithmic_bytes(model) * nshots * steps / (tb / 1e3) / 1e9
    return {"shots": nshots, "steps": steps, "ricker_hz": "U[10, 25], seed 2",
            "value": round(cells / (tb / 1e3) / 1e9, 3), "unit": "Gcell/s",
            "shot_steps_per_s": round(nshots * steps / (tb / 1e3), 1),
            "per_shot_loop_gcells": round(cells / (loop_ms / 1e3) / 1e9, 3),
            "speedup_vs_per_shot_loop": round(loop_ms / tb, 3),
            "seg_rows": {"batch": tile_b, "per_shot": tile_1},
            "roofline": {"bytes": "coefficients read once per segment for all shots",
                         "achieved_gbs": round(shared, 1), "frac": round(shared / peak, 4),
                         "frac_if_unshared": round(unshared / peak, 4)}}


def uneven_rate(mfdm, device: int, nmodels: int = 32, steps: int = 128):
    """Cell-steps/s of `nmodels` layered models of seeded uneven sizes (nx
    400..2000, nz 300..1000, seed 3) stepped together as one group (one
    captured graph, the models on parallel branches) against the same models
    stepped one after another, each through its own captured graph. Every model
    gets its segment height from the autotuner first; device time (CUDA events)."""
    models = modelgen.uneven_models(nmodels, seed=3, nt=10)
    solvers = [mfdm.Solver.from_model(m, device=device) for m in models]
    try:
        tiles = [s.autotune() for s in solvers]
        loop_ms = 0.0
        for s in solvers:
            s.set_shot(0, reset=True)
            s.step(32)  # warm-up, graph capture
            t, _ = s.time_steps(steps)
            loop_ms += t
        for s in solvers:
            s.set_shot(0, reset=True)
        with mfdm.Group(solvers) as g:
            g.step(32)
            tg = g.time_steps(steps)
    finally:
        for s in solvers:
            s.close()
    cells = sum(m.cells for m in models) * steps
    peak, _ = peaks()
    gbs = sum(algorithmic_bytes(m) for m in models) * steps / (tg / 1e3) / 1e9
    return {"models": nmodels, "steps": steps, "cells": sum(m.cells for m in models),
            "value": round(cells / (tg / 1e3) / 1e9, 3), "unit": "Gcell/s",
            "model_loop_gcells": round(cells / (loop_ms / 1e3) / 1e9, 3),
            "speedup_vs_model_loop": round(loop_ms / tg, 3),
            "seg_rows": {str(r): tiles.count(r) for r in sorted(set(tiles))},
            "roofline": {"achieved_gbs": round(gbs, 1), "frac": round(gbs / peak, 4)}}


def adjoint_rate(mfdm, device: int, nsteps: int = 4000, every: int = 50, repeats: int = 3):
    """Cost of the adjoint-state gradient against a plain forward run on the
    800x400 curvilinear model pair (4000 RK4 steps, checkpoint every 50): host
    wall time of the synchronous calls. The observed records come from the true
    model (+10 % vs Gaussian anomaly); the gradient is that of the L2 misfit
    of the smoothed initial model's records against them. The adjoint's
    forward pass (with checkpoints) plus its backward pass is compared with
    mfdm_step over the same steps; the one-time operator assembly is listed
    separately. Each pass runs `repeats` times and the median is reported,
    with every run listed (the backward enqueues ~40 host calls a step, so a
    busy host can slow a single run)."""
    true, m = modelgen.adjoint_pair(800, 400, nt=nsteps)
    with mfdm.Solver.from_model(true, device=device) as st:
        st.set_shot(0, reset=True)
        st.step(nsteps)
        obs = st.records()
    with mfdm.Solver.from_model(m, device=device) as s:
        s.set_shot(0, reset=True)
        s.step(64)
        fwds, afwds, bwds = [], [], []
        for _ in range(repeats):
            s.set_shot(0, reset=True)
            t0 = time.perf_counter()
            s.step(nsteps)
            fwds.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        s.adjoint_forward(nsteps, every)  # first call also assembles the operators
        first = time.perf_counter() - t0
        for _ in range(repeats):
            t0 = time.perf_counter()
            rec = s.adjoint_forward(nsteps, every)
            afwds.append(time.perf_counter() - t0)
            res = {k: (rec[k] - obs[k]).astype(np.float32) for k in rec}
            t0 = time.perf_counter()
            grad = s.adjoint_backward(res)
            bwds.append(time.perf_counter() - t0)
        misfit = 0.5 * sum(float(np.sum(np.float64(r) ** 2)) for r in res.values())
        fwd, afwd, bwd = (statistics.median(v) for v in (fwds, afwds, bwds))
        # the same with every segment's stage inputs kept in device memory
        # (no recompute; 4 * 4000 states of this model, about 85 GB of HBM)
        s.adjoint_memory(150 * 10 ** 9)
        t0 = time.perf_counter()
        s.adjoint_forward(nsteps, every)  # first: allocates the keep buffer, encodes its maps
        kfirst = time.perf_counter() - t0
        kfwds, kbwds = [], []
        for _ in range(repeats):
            t0 = time.perf_counter()
            s.adjoint_forward(nsteps, every)
            kfwds.append(time.perf_counter() - t0)
            t0 = time.perf_counter()
            s.adjoint_backward(res)
            kbwds.append(time.perf_counter() - t0)
        kfwd, kbwd = statistics.median(kfwds), statistics.median(kbwds)
        s.adjoint_memory(0)
    # where the vs anomaly sits: the solid C55 gradient should be largest near it
    g55 = np.abs(grad["C55"])
    iz, ix = np.unravel_index(int(np.argmax(g55)), g55.shape)
    return {"model": "curvilinear 800x400, true (+10 % vs anomaly) / smoothed initial",
            "steps": nsteps, "ckpt_every": every, "misfit": float(f"{misfit:.6e}"),
            "max_abs_dC55_at": [int(iz), int(ix)],
            "forward_s": round(fwd, 4), "adjoint_forward_s": round(afwd, 4),
            "backward_s": round(bwd, 4), "assembly_s": round(first - afwd, 4),
            "adjoint_over_forward": round((afwd + bwd) / fwd, 3),
            "runs": {"forward_s": [round(v, 4) for v in fwds],
                     "adjoint_forward_s": [round(v, 4) for v in afwds],
                     "backward_s": [round(v, 4) for v in bwds],
                     "kept_backward_s": [round(v, 4) for v in kbwds], "statistic": "median"},
            "kept_segments": {"adjoint_forward_s": round(kfwd, 4), "backward_s": round(kbwd, 4),
                              "keep_setup_s": round(kfirst - kfwd, 4),
                              "adjoint_over_forward": round((kfwd + kbwd) / fwd, 3)}}


def adjoint_4096x2048_rate(mfdm, device: int, nsteps: int = 400, every: int = 50):
    """Adjoint cost at the 4096x2048 curvilinear size: `nsteps` RK4 steps,
    checkpoint every `every`, every segment recomputed (one level, the next
    segment recomputed into a second stage-input buffer while the current one
    is reversed). Residuals: 1 % of the model's own records. Host wall time of
    the synchronous calls, the second of two adjoint passes (the first also
    assembles the transposed operators)."""
    import torch
    m = modelgen.curvilinear_4096x2048(nt=nsteps)
    torch.cuda.synchronize(device)
    free0, _ = torch.cuda.mem_get_info(device)
    with mfdm.Solver.from_model(m, device=device) as s:
        s.set_shot(0, reset=True)
        s.step(16)
        s.set_shot(0, reset=True)
        t0 = time.perf_counter()
        s.step(nsteps)
        fwd = time.perf_counter() - t0
        s.set_shot(0, reset=True)
        rec = s.adjoint_forward(nsteps, every)
        s.adjoint_backward_only({k: (0.01 * v).astype(np.float32) for k, v in rec.items()})
        s.set_shot(0, reset=True)
        t0 = time.perf_counter()
        rec = s.adjoint_forward(nsteps, every)
        afwd = time.perf_counter() - t0
        t0 = time.perf_counter()
        s.adjoint_backward_only({k: (0.01 * v).astype(np.float32) for k, v in rec.items()})
        bwd = time.perf_counter() - t0
        used = free0 - torch.cuda.mem_get_info(device)[0]
    return {"model": "curvilinear 4096x2048", "steps": nsteps, "ckpt_every": every,
            "forward_s": round(fwd, 4), "adjoint_forward_s": round(afwd, 4),
            "backward_s": round(bwd, 4), "adjoint_over_forward": round((afwd + bwd) / fwd, 3),
            "device_gb_in_use": round(used / 1e9, 2)}


def large_adjoint_rate(mfdm, device: int, nshots: int = 1, nsteps: int = 200, every: int = 100,
                       inner: int = 5, ckpt_probe_steps: int = 0):
    """The 8192 x 4096 batched-adjoint workload (von Kármán rough seafloor, Hurst
    0.7, rms 20 m, correlation 200 m, seed 5; 16 sources, 10 Hz) at a reduced
    step count: `nshots` of its shots one after another on one handle, two
    checkpoint levels (a state every `every` steps; the backward pass re-runs
    each segment keeping a state every `inner` steps), the L2 misfit of the
    records against zero observations, gradients summed on the device in FP32.
    Host wall time of the synchronous calls; device memory in use measured with
    cudaMemGetInfo after each shot (its largest value, minus what was in use
    before the handle opened). With ckpt_probe_steps > 0 an adjoint forward
    pass of that many steps also measures the memory of its checkpoints."""
    import torch
    m = modelgen.rough_seafloor(8192, 4096, nt=nsteps)
    torch.cuda.synchronize(device)
    free0, total = torch.cuda.mem_get_info(device)
    peak, shots_s = 0, []
    with mfdm.Solver.from_model(m, device=device) as s:
        info = s.info()
        s.set_shot(0, reset=True)
        s.step(8)
        s.set_shot(0, reset=True)
        t0 = time.perf_counter()
        s.step(nsteps)
        fwd = time.perf_counter() - t0
        s.adjoint_inner(inner)
        acc = torch.zeros((2 * info["nz_f"] + 5 * info["nz_s"]) * info["nx"], dtype=torch.float32,
                          device=f"cuda:{device}")
        s.set_shot(0, reset=True)
        t0 = time.perf_counter()
        s.adjoint_forward(nsteps, every)  # first call: operator assembly
        first = time.perf_counter() - t0
        for shot in range(nshots):
            s.set_shot(shot, reset=True)
            t0 = time.perf_counter()
            rec = s.adjoint_forward(nsteps, every)
            t1 = time.perf_counter()
            s.adjoint_backward_only(rec)
            s.adjoint_accumulate_grad(acc)
            torch.cuda.synchronize(device)
            t2 = time.perf_counter()
            peak = max(peak, free0 - torch.cuda.mem_get_info(device)[0])
            shots_s.append((t1 - t0, t2 - t1))
        probe = None
        if ckpt_probe_steps > 0:
            s.set_shot(0, reset=True)
            t0 = time.perf_counter()
            s.adjoint_forward(ckpt_probe_steps, every)
            probe = {"steps": ckpt_probe_steps, "adjoint_forward_s": round(time.perf_counter() - t0, 3),
                     "device_gb_in_use": round((free0 - torch.cuda.mem_get_info(device)[0]) / 1e9, 2)}
    afwd = statistics.median(a for a, _ in shots_s)
    bwd = statistics.median(b for _, b in shots_s)
    return {"model": "rough seafloor 8192x4096 (von Karman H 0.7, rms 20 m, corr 200 m, seed 5), "
                     "16 sources, 10 Hz", "cells": m.cells, "shots_run": nshots, "steps": nsteps,
            "ckpt_every": every, "inner_every": inner, "forward_s": round(fwd, 4),
            "assembly_s": round(first - afwd, 3), "adjoint_forward_s": round(afwd, 4),
            "backward_s": round(bwd, 4), "adjoint_over_forward": round((afwd + bwd) / fwd, 3),
            "device_gb_peak": round(peak / 1e9, 2), "device_gb_total": round(total / 1e9, 1),
            "grad_abs_max": float(f"{float(acc.abs().max()):.4e}"),
            "checkpoint_probe": probe}


def solid_only_rate(mfdm, device: int, n: int = 2048, steps: int = 256):
    """Solid only with a free surface (calc_type 0) on an n x n grid with surface
    topography: device time of `steps` graph-captured steps, and the whole
    step's share of the HBM roofline at the solid's algorithmic 464 B per
    cell-step (16 state + 4 x 9 coefficient floats x 4 B)."""
    m = modelgen.make_solid_model(n, n, npd=20, fpeak=15.0, dt=5e-4, nt=10, src_x=[n // 2],
                                  src_z=[20], amp=20.0, wavelength=600.0)
    with mfdm.SolidSolver.from_model(m, device=device) as s:
        s.set_shot(0, reset=True)
        s.step(32)
        ms = s.time_steps(steps)
        # FP64 error: 40 steps from rest against the FP64 solid-only oracle
        from oracle import pyoracle
        pyoracle.build()
        s.set_shot(0, reset=True)
        s.step(40)
        names = ("solid_vx", "solid_vz", "solid_sx", "solid_sz", "solid_sxz")
        ours = [s.field(k) for k in names]
    ref = pyoracle.forward_solid(m, 40, pyoracle.record_gap(m.dt), 64, final_fields=True)
    errs = {k: rel_l2(a, b) for k, a, b in zip(names, ours, ref["solid"])}
    worst = max(errs, key=errs.get)
    gcells = m.cells * steps / (ms / 1e3) / 1e9
    gbs = m.cells * 464 * steps / (ms / 1e3) / 1e9
    peak, _ = peaks()
    return {"grid": f"{n}x{n}", "steps": steps, "value": round(gcells, 3), "unit": "Gcell/s",
            "ms_per_step": round(ms / steps, 4), "achieved_gbs": round(gbs, 1),
            "frac_of_measured_hbm": round(gbs / peak, 4),
            "fp64_error": {"rel_l2": float(f"{errs[worst]:.3e}"), "field": worst, "steps": 40}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="only the warm-up and timed steps (a short launch list for ncu)")
    ap.add_argument("--blocks-per-sm", type=int, default=0, choices=[0, 2, 3, 4],
                    help="stage kernel build (0: the default, as for any model)")
    ap.add_argument("--seg-rows", type=int, default=0,
                    help="rows per segment block of the stage launches (0: the default for the grid)")
    ap.add_argument("--adjoint-profile", action="store_true",
                    help="only a short adjoint run on a curvilinear model (16 steps, checkpoint "
                         "every 8, seeded residuals): a launch list of the adjoint kernels for ncu")
    ap.add_argument("--adjoint-grid", type=int, nargs=2, default=[800, 400], metavar=("NX", "NZ"),
                    help="grid of --adjoint-profile (default 800 400)")
    ap.add_argument("--large-adjoint", type=int, nargs=5, default=None,
                    metavar=("SHOTS", "STEPS", "EVERY", "INNER", "PROBE"),
                    help="only the 8192x4096 rough-seafloor adjoint: SHOTS shots of STEPS steps, "
                         "checkpoints every EVERY / INNER steps, and a PROBE-step checkpoint "
                         "memory probe (0: none)")
    ap.add_argument("--solid-profile", type=int, default=0, metavar="N",
                    help="only a short solid-only run on an N x N model (3 + 8 steps): a launch "
                         "list of the solid-only kernels for ncu")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.large_adjoint:
        mfdm = importlib.import_module("marineseis-fdm-2d_b200")
        mfdm.load_library()
        sh, st, ev, inn, pr = args.large_adjoint
        print(json.dumps({"large_adjoint": large_adjoint_rate(mfdm, 0, sh, st, ev, inn, pr)}))
        return

    if args.solid_profile:
        mfdm = importlib.import_module("marineseis-fdm-2d_b200")
        mfdm.load_library()
        n = args.solid_profile
        m = modelgen.make_solid_model(n, n, npd=20, fpeak=15.0, dt=5e-4, nt=10, src_x=[n // 2],
                                      src_z=[20], amp=20.0, wavelength=600.0)
        with mfdm.SolidSolver.from_model(m) as s:
            s.set_shot(0, reset=True)
            s.step(3)
            ms = s.time_steps(8)
        print(json.dumps({"solid_profile_run": True, "grid": f"{n}x{n}", "ms_per_step": ms / 8}))
        return

    if args.adjoint_profile:
        mfdm = importlib.import_module("marineseis-fdm-2d_b200")
        mfdm.load_library()
        m = modelgen.curvilinear(args.adjoint_grid[0], args.adjoint_grid[1], nt=16)
        with mfdm.Solver.from_model(m) as s:
            s.set_shot(0, reset=True)
            rec = s.adjoint_forward(16, 8)
            rng = np.random.default_rng(1)
            g = s.adjoint_backward({k: rng.standard_normal(v.shape).astype(np.float32)
                                    for k, v in rec.items()})
        print(json.dumps({"adjoint_profile_run": True, "max_abs_dC11": float(np.abs(g["C11"]).max())}))
        return
    world, rank, local, dist = dist_setup(args)
    model = WORKLOADS[args.workload]()
    if args.impl == "reference":
        run_reference(args, model, world, rank)
        if dist is not None:
            dist.destroy_process_group()
        return

    mfdm = importlib.import_module("marineseis-fdm-2d_b200")
    mfdm.load_library()
    solver = mfdm.Solver.from_model(model, device=local)
    solver.set_blocks_per_sm(args.blocks_per_sm)
    solver.set_tile(args.seg_rows)
    solver.set_shot(0, reset=True)
    solver.step(args.warmup)

    # ---- timed region: K steps through the captured time loop ----
    barrier(dist, local)
    with ClockSampler(local) as clk:
        total_ms, _ = solver.time_steps(args.steps)
    ms = max_over_ranks(dist, total_ms, local)
    secs = ms / 1e3
    value = world * model.cells * args.steps / secs / 1e9
    if args.profile:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": round(value, 3), "unit": "Gcell/s",
                              "steps": args.steps, "warmup": args.warmup,
                              "config": {"workload": args.workload}, "profile_run": True}))
        solver.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    # ---- per-kernel durations (events around every launch) ----
    nk = min(args.steps, 200)
    _, kms = solver.time_steps(nk, per_kernel=True)
    stage_ms = sum(kms[:4]) / nk  # the four stage launches of one step
    alg = algorithmic_bytes(model)
    peak, peak_kind = peaks()
    achieved = alg / (stage_ms / 1e3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "stage_kernel_traffic.json")
    if os.path.exists(tp):
        tj = json.load(open(tp))
        if tj.get("workload") == args.workload:
            traffic = tj.get("dram_bytes_per_launch")

    # ---- end to end through the public API with host buffers ----
    import torch
    pinned = {}
    for grp in ("fluid", "solid", "metric"):
        for k, v in getattr(model, grp).items():
            t = torch.empty(v.shape, dtype=torch.float32, pin_memory=True)
            t.numpy()[...] = v
            pinned[(grp, k)] = t
    host_model = modelgen.Model(**{f: getattr(model, f) for f in (
        "nx", "nz_f", "nz_s", "h", "fpeak", "dt", "nt", "snapshot", "src_x", "src_z", "npd",
        "npow", "thickness", "vp_max", "rc", "beta0")})
    for (grp, k), t in pinned.items():
        getattr(host_model, grp)[k] = t.numpy()
    h2d = sum(t.numel() * 4 for (grp, k), t in pinned.items()
              if k in ("K", "rho", "C11", "C13", "C33", "C55", "J", "xi_x", "xi_z", "ze_x", "ze_z"))
    # one untimed upload first: on some hosts the first transfer from freshly
    # pinned pages took 0.33 s instead of 7 ms (the timed pass uploads again)
    solver.load_model(host_model)
    barrier(dist, local)
    t0 = time.perf_counter()
    solver.load_model(host_model)
    solver.set_shot(0, reset=True)
    t1 = time.perf_counter()
    solver.step(args.steps)
    t2 = time.perf_counter()
    rec = solver.records()
    t3 = time.perf_counter()
    e2e_s = t3 - t0
    e2e_parts = {"upload_s": round(t1 - t0, 4), "steps_s": round(t2 - t1, 4),
                 "records_s": round(t3 - t2, 4)}
    e2e_s = max_over_ranks(dist, e2e_s, local)
    d2h = sum(a.nbytes for a in rec.values())
    e2e = world * model.cells * args.steps / e2e_s / 1e9

    # ---- CPU baseline (rank 0, single GPU runs only) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, threads, n, s = cpu_oracle_rate(model, target_s=15.0, max_steps=50)
        cpu = {"value": round(rate, 5), "unit": "Gcell/s", "cores": threads, "kind": "port",
               "sample": f"{n} RK4 steps of {args.workload} in {s:.1f} s (FP32 oracle, OpenMP)"}

    # the other workloads, for context, on single-GPU runs only (a multi-GPU run
    # would hold every GPU while rank 0 alone works through them)
    other = {}
    if rank == 0 and world == 1 and args.workload == DEFAULT_WORKLOAD:
        small = modelgen.curvilinear_1200x800(nt=10)
        with mfdm.Solver.from_model(small, device=local) as s2:
            s2.set_shot(0, reset=True)
            s2.step(args.warmup)
            n2 = max(args.steps, 200)
            t2, _ = s2.time_steps(n2)
            other["curvilinear_1200x800"] = {
                "value": round(small.cells * n2 / (t2 / 1e3) / 1e9, 3), "unit": "Gcell/s",
                "ms_per_step": round(t2 / n2, 4)}
        other["curvilinear_1200x800"]["fp64_error"] = fp64_error(mfdm, small, 300, local)
        other["batched_1200x800_64_shots"] = batched_rate(mfdm, small, local, args.warmup)
        other["batched_1200x800_64_shots"]["fp64_error"] = dict(
            fp64_error(mfdm, small, 300, local, shot=batched_shots(small, 64)[0]),
            note="shot 0 with its own frequency; every batched shot is bit-identical to "
                 "the same shot run alone (tests/test_gpu_batch.py)")
        other["uneven_32_models"] = uneven_rate(mfdm, local)
        m0 = modelgen.uneven_models(1, seed=3, nt=10)[0]
        other["uneven_32_models"]["fp64_error"] = dict(
            fp64_error(mfdm, m0, 200, local),
            note="model 0; every grouped model is bit-identical to the model stepped alone")
        other["adjoint_800x400"] = adjoint_rate(mfdm, local)
        _, m_init = modelgen.adjoint_pair(800, 400, nt=10)
        other["adjoint_800x400"]["fp64_error"] = dict(
            fp64_error(mfdm, m_init, 400, local),
            note="forward state of the initial model; the gradient against the FP64 "
                 "adjoint oracle is checked in tests/test_gpu_adjoint.py (rel-L2 <= 1e-3)")
        other["adjoint_4096x2048"] = adjoint_4096x2048_rate(mfdm, local)
        other["solid_only_2048x2048"] = solid_only_rate(mfdm, local)
        other["adjoint_8192x4096_rough_seafloor"] = large_adjoint_rate(mfdm, local)
        other["reference_cuda_build"] = reference_cuda_build([
            ("curvilinear_4096x2048", lambda nt: modelgen.curvilinear_4096x2048(nt=nt),
             (100, 1100), (200, 5200)),
            ("curvilinear_1200x800", lambda nt: modelgen.curvilinear_1200x800(nt=nt),
             (500, 4500), (1000, 21000))])
        # the same against this library's device-timed step (CUDA events), which
        # carries no process start-up jitter
        dev_ms = {"curvilinear_4096x2048": ms / args.steps,
                  "curvilinear_1200x800": other["curvilinear_1200x800"]["ms_per_step"]}
        for name, row in other["reference_cuda_build"].items():
            if isinstance(row, dict) and name in dev_ms and "reference" in row:
                row["library_device_ms_per_step"] = round(dev_ms[name], 4)
                row["speedup_device_timed"] = round(row["reference"]["ms_per_step"] / dev_ms[name], 2)

    clocks = clk.summary()
    solver.close()
    fp64 = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        fp64 = fp64_error(mfdm, model, 40, local)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Gcell/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator, no dataset)",
            "config": bench_config(args, model, world),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                         "peak_kind": peak_kind,
                         "algorithmic_bytes_per_step": alg,
                         "stage_launch_ms": [round(k / nk, 5) for k in kms[:4]],
                         "filter_launch_ms": round(kms[4] / nk, 5)},
            "gpu_launches": 5 * args.steps,
            "e2e": {"value": round(e2e, 3), "unit": "Gcell/s",
                    "h2d_bytes_per_step": int(h2d // args.steps),
                    "d2h_bytes_per_step": int(d2h // args.steps), **e2e_parts},
            "cpu_baseline": cpu,
            "fp64_error": fp64,
            "clocks": clocks,
            "other_workloads": other,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
