"""Regenerates the golden fixtures from the reference's own CUDA build.

Needs a GPU and oracle/_ref/main_debug (built by `make -C oracle ref` from the
reference sources). For every case in cases.py it writes the model, runs
`main_debug <model.json> <out>` twice, and stores the records (and, for the
small cases, the last snapshot) of the first run in tests/golden/<case>.npz,
plus the largest relative L2 difference between the two runs (the reference's
own run-to-run spread; its in-place interface filter races across blocks).

    python tests/golden/make_golden.py [case ...] [--work DIR]
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import cases  # noqa: E402

REF_BIN = os.path.join(cases.ROOT, "oracle", "_ref", "main_debug")


def run_reference(jpath: str, out: str) -> float:
    t0 = time.time()
    subprocess.run([REF_BIN, jpath, out], check=True, stdout=subprocess.DEVNULL)
    return time.time() - t0


def load_records(out: str, nx: int):
    rec = {}
    for key, fname in (("svx", "solid_vx.bin"), ("svz", "solid_vz.bin"), ("fp", "fluid_p.bin")):
        a = np.fromfile(os.path.join(out, "0", "record", fname), dtype="<f4")
        rec[key] = a.reshape(-1, nx)
    return rec


def load_snapshot(out: str, it: int, model):
    snap = {}
    for medium, rows in (("solid", model.nz_s), ("fluid", model.nz_f)):
        for comp in ("vx", "vz"):
            p = os.path.join(out, "0", "snapshot", medium, comp, f"{comp}_{it:06d}.bin")
            snap[f"{medium}_{comp}"] = np.fromfile(p, dtype="<f4").reshape(rows, model.nx)
    return snap


def rel(a, b):
    d = np.linalg.norm(np.asarray(b, np.float64))
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / d) if d > 0 else 0.0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("names", nargs="*")
    ap.add_argument("--work", default=os.path.join(cases.ROOT, "gpurun_out", "golden_work"))
    ap.add_argument("--outdir", default=cases.GOLDEN_DIR)
    args = ap.parse_args()
    names = args.names or list(cases.CASES)
    summary = {}
    for name in names:
        build, stride, keep_snap = cases.CASES[name]
        model = build()
        if keep_snap:
            model.snapshot = model.nt - 1  # snapshots at it = 0 and it = nt - 1
        work = os.path.join(args.work, name)
        jpath = cases.modelgen.write_model(model, os.path.join(work, "model"))
        outs = [os.path.join(work, "out_a"), os.path.join(work, "out_b")]
        secs = [run_reference(jpath, o) for o in outs]
        ra, rb = load_records(outs[0], model.nx), load_records(outs[1], model.nx)
        spread = max(rel(ra[k], rb[k]) for k in ra)
        data = {k: ra[k][:, ::stride].astype(np.float32) for k in ra}
        data["receiver_stride"] = np.int32(stride)
        data["nt"] = np.int32(model.nt)
        data["run_to_run_rel_l2"] = np.float64(spread)
        if keep_snap:
            sa = load_snapshot(outs[0], model.nt - 1, model)
            sb = load_snapshot(outs[1], model.nt - 1, model)
            for k in sa:
                data["snap_" + k] = sa[k]
            data["snap_run_to_run_rel_l2"] = np.float64(max(rel(sa[k], sb[k]) for k in sa))
        os.makedirs(args.outdir, exist_ok=True)
        np.savez_compressed(os.path.join(args.outdir, name + ".npz"), **data)
        summary[name] = {"seconds": secs, "run_to_run_rel_l2": spread,
                         "samples": int(ra["svx"].shape[0])}
        print(name, json.dumps(summary[name]), flush=True)
        shutil.rmtree(work, ignore_errors=True)
    with open(os.path.join(args.outdir, "golden_summary.json"), "w") as f:
        json.dump(summary, f, indent=1)


if __name__ == "__main__":
    main()
