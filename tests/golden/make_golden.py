"""Regenerates the golden fixtures from the reference's own CUDA build.

Needs a GPU and oracle/_ref/main_debug (built by `make -C oracle ref` from the
reference sources). For every case in cases.py it writes the model, runs
`main_debug <model.json> <out>` twice, and stores the records (and the last
snapshot, whole or every k-th row and column) of the first run in
tests/golden/<case>.npz, plus the largest relative L2 difference between the
two runs (the reference's own run-to-run spread; its in-place interface filter
races across blocks). For the long cases (cases.NOFMA_CASES) it also runs
oracle/_ref/main_debug_nofma (`make -C oracle ref-nofma`: the same sources
with FMA contraction off) and stores each record set's relative L2 distance
between the two builds, the FP32 noise floor of the scheme at that length.

    python tests/golden/make_golden.py [case ...] [--work DIR] [--outdir DIR]
    python tests/golden/make_golden.py --fp64 [case ...]   (CPU: FP64 oracle records)
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import cases  # noqa: E402

REF_BIN = os.path.join(cases.ROOT, "oracle", "_ref", "main_debug")
REF_NOFMA_BIN = os.path.join(cases.ROOT, "oracle", "_ref", "main_debug_nofma")
FP64_STRIDE = 16  # receiver stride of the stored FP64 oracle records (at least the case's)


def run_reference(jpath: str, out: str, binary: str = REF_BIN) -> float:
    t0 = time.time()
    subprocess.run([binary, jpath, out], check=True, stdout=subprocess.DEVNULL)
    return time.time() - t0


def load_records(out: str, nx: int, solid_only: bool = False):
    rec = {}
    files = (("svz", "solid_vz.bin"),) if solid_only else (
        ("svx", "solid_vx.bin"), ("svz", "solid_vz.bin"), ("fp", "fluid_p.bin"))
    for key, fname in files:
        a = np.fromfile(os.path.join(out, "0", "record", fname), dtype="<f4")
        rec[key] = a.reshape(-1, nx)
    return rec


def load_snapshot(out: str, it: int, model):
    snap = {}
    media = ((("solid", model.nz),) if isinstance(model, cases.modelgen.SolidModel)
             else (("solid", model.nz_s), ("fluid", model.nz_f)))
    for medium, rows in media:
        for comp in ("vx", "vz"):
            p = os.path.join(out, "0", "snapshot", medium, comp, f"{comp}_{it:06d}.bin")
            snap[f"{medium}_{comp}"] = np.fromfile(p, dtype="<f4").reshape(rows, model.nx)
    return snap


def rel(a, b):
    d = np.linalg.norm(np.asarray(b, np.float64))
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / d) if d > 0 else 0.0


def add_fp64_records(name: str, outdir: str):
    """Adds the FP64 oracle's records (every FP64_STRIDE-th receiver) to an existing fixture.

    Runs on the CPU. Over long runs the FP32 rounding noise of this scheme grows
    above 1e-5 (the reference build itself drifts from the FP64 solution), so
    the fixture also stores the FP64 records that both FP32 implementations are
    measured against."""
    sys.path.insert(0, cases.ROOT)
    from oracle import pyoracle
    build, stride, _ = cases.CASES[name]
    model = build()
    path = os.path.join(outdir, name + ".npz")
    data = dict(np.load(path))
    nt = int(data["nt"])
    r = pyoracle.forward(model, nt, pyoracle.record_gap(model.dt), 64)
    s64 = max(stride, FP64_STRIDE)
    sub = s64 // stride
    data["fp64_stride"] = np.int32(s64)
    for k in ("svx", "svz", "fp"):
        # stored in float32: the rounding (< 1e-7 relative) is far below what is compared
        data["fp64_" + k] = r[k][:, ::s64].astype(np.float32)
    data["fp64_ref_rel_l2"] = np.float64(max(rel(data[k][:, ::sub], data["fp64_" + k])
                                             for k in ("svx", "svz", "fp")))
    np.savez_compressed(path, **data)
    print(name, "reference build vs FP64 oracle:", float(data["fp64_ref_rel_l2"]), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("names", nargs="*")
    ap.add_argument("--fp64", action="store_true",
                    help="add FP64 oracle records to existing fixtures (CPU only)")
    ap.add_argument("--work", default=os.path.join(tempfile.gettempdir(), "mfdm_golden_work"))
    ap.add_argument("--outdir", default=cases.GOLDEN_DIR)
    ap.add_argument("--no-nofma", action="store_true", help="skip the FMA-off reference build")
    args = ap.parse_args()
    names = args.names or list(cases.CASES)
    if args.fp64:
        for name in names:
            add_fp64_records(name, args.outdir)
        return
    summary = {}
    for name in names:
        build, stride, keep_snap = cases.CASES[name]
        step = cases.snapshot_step(keep_snap)
        model = build()
        if step:
            model.snapshot = model.nt - 1  # snapshots at it = 0 and it = nt - 1
        work = os.path.join(args.work, name)
        jpath = cases.modelgen.write_model(model, os.path.join(work, "model"))
        outs = [os.path.join(work, "out_a"), os.path.join(work, "out_b")]
        secs = [run_reference(jpath, o) for o in outs]
        solid_only = isinstance(model, cases.modelgen.SolidModel)
        ra = load_records(outs[0], model.nx, solid_only)
        rb = load_records(outs[1], model.nx, solid_only)
        spread = max(rel(ra[k], rb[k]) for k in ra)
        data = {k: ra[k][:, ::stride].astype(np.float32) for k in ra}
        data["receiver_stride"] = np.int32(stride)
        data["nt"] = np.int32(model.nt)
        data["run_to_run_rel_l2"] = np.float64(spread)
        entry = {"seconds": secs, "run_to_run_rel_l2": spread, "samples": int(ra["svz"].shape[0])}
        if name in cases.NOFMA_CASES and not args.no_nofma:
            out_c = os.path.join(work, "out_nofma")
            entry["seconds_nofma"] = run_reference(jpath, out_c, REF_NOFMA_BIN)
            rc = load_records(out_c, model.nx, solid_only)
            for k in ra:
                data["nofma_rel_l2_" + k] = np.float64(rel(rc[k], ra[k]))
                entry["nofma_rel_l2_" + k] = float(data["nofma_rel_l2_" + k])
        if step:
            data["snapshot_step"] = np.int32(step)
            sa = load_snapshot(outs[0], model.nt - 1, model)
            sb = load_snapshot(outs[1], model.nt - 1, model)
            for k in sa:
                data["snap_" + k] = np.ascontiguousarray(sa[k][::step, ::step])
            data["snap_run_to_run_rel_l2"] = np.float64(max(rel(sa[k], sb[k]) for k in sa))
        os.makedirs(args.outdir, exist_ok=True)
        np.savez_compressed(os.path.join(args.outdir, name + ".npz"), **data)
        summary[name] = entry
        print(name, json.dumps(summary[name]), flush=True)
        shutil.rmtree(work, ignore_errors=True)
    sp = os.path.join(args.outdir, "golden_summary.json")
    if not os.path.exists(sp) and os.path.exists(os.path.join(cases.GOLDEN_DIR, "golden_summary.json")):
        sp0 = os.path.join(cases.GOLDEN_DIR, "golden_summary.json")
        merged = json.load(open(sp0))
    else:
        merged = json.load(open(sp)) if os.path.exists(sp) else {}
    merged.update(summary)
    with open(sp, "w") as f:
        json.dump(merged, f, indent=1)


if __name__ == "__main__":
    main()
