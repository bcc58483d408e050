"""Times the reference's own CUDA build against this library on the same model.

Needs a GPU and oracle/_ref/main_debug (built by `make -C oracle ref` from the
reference sources). For each workload the same JSON model runs through the
reference build and through this library's drop-in CLI (bin/main_debug), at two
step counts each (three interleaved runs of each); the per-step time is the
difference of the median wall times over the difference of the step counts,
so start-up, model loading and file output cancel. Snapshots are disabled (snapshot > nt); receiver records are
written by both, as the reference does.

    python tests/golden/time_reference.py [--work DIR] [workload ...]
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import cases  # noqa: E402

REF_BIN = os.path.join(cases.ROOT, "oracle", "_ref", "main_debug")
OUR_BIN = os.path.join(cases.ROOT, "marineseis-fdm-2d_b200", "bin", "main_debug")
REPEATS = 3

# workload -> (model builder, short run, long run)
WORKLOADS = {
    "curvilinear_1200x800": (lambda nt: cases.modelgen.curvilinear_1200x800(nt=nt), 500, 8500),
    "curvilinear_4096x2048": (lambda nt: cases.modelgen.curvilinear_4096x2048(nt=nt), 200, 2200),
}


def wall(binary: str, jpath: str, out: str) -> float:
    t0 = time.perf_counter()
    subprocess.run([binary, jpath, out], check=True, stdout=subprocess.DEVNULL)
    return time.perf_counter() - t0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("names", nargs="*")
    ap.add_argument("--work", default=os.path.join(tempfile.gettempdir(), "mfdm_time_reference"))
    args = ap.parse_args()
    result = {}
    for name in args.names or list(WORKLOADS):
        build, n1, n2 = WORKLOADS[name]
        paths = {}
        for nt in (n1, n2):
            model = build(nt)
            model.snapshot = nt + 1
            work = os.path.join(args.work, f"{name}_{nt}")
            paths[nt] = (work, cases.modelgen.write_model(model, os.path.join(work, "model")))
        cells = model.cells
        row = {}
        for label, binary in (("reference", REF_BIN), ("library", OUR_BIN)):
            wall(binary, paths[n1][1], os.path.join(paths[n1][0], "out"))  # page the files in
            # short and long runs interleaved, so drifts in start-up cost hit both
            runs = {n1: [], n2: []}
            for _ in range(REPEATS):
                for nt in (n1, n2):
                    runs[nt].append(wall(binary, paths[nt][1], os.path.join(paths[nt][0], "out")))
            ms = (statistics.median(runs[n2]) - statistics.median(runs[n1])) / (n2 - n1) * 1e3
            row[label] = {"ms_per_step": round(ms, 4), "gcells": round(cells / (ms / 1e3) / 1e9, 3),
                          "wall_s": {str(k): [round(x, 3) for x in v] for k, v in runs.items()}}
        for nt in (n1, n2):
            shutil.rmtree(paths[nt][0], ignore_errors=True)
        row["speedup"] = round(row["reference"]["ms_per_step"] / row["library"]["ms_per_step"], 2)
        row["steps"] = [n1, n2]
        result[name] = row
        print(name, json.dumps(row), flush=True)
    os.makedirs(args.work, exist_ok=True)
    with open(os.path.join(args.work, "summary.json"), "w") as f:
        json.dump(result, f, indent=1)


if __name__ == "__main__":
    main()
