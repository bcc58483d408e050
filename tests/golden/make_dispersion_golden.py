"""Golden vectors of the reference's dispersion imaging and mode curves.

Imports `dispersion_imaging` and `omega_from_c` from the reference's
tools/test.py (a plain numpy module; its plotting code only runs from its
__main__) and evaluates them on a seeded synthetic gather: a sum of two
dispersive wave trains plus noise, 256 samples at 1 kHz on 48 traces 4 m
apart. The gather is passed in float64, so the reference computes in FP64.
Writes tests/golden/dispersion_small.npz.

    python tests/golden/make_dispersion_golden.py [--reference DIR]
"""
from __future__ import annotations

import argparse
import importlib.util
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def synthetic_gather(nt=256, ntr=48, fs=1000.0, dx=4.0, seed=11):
    rng = np.random.default_rng(seed)
    t = np.arange(nt) / fs
    x = 10.0 + dx * np.arange(ntr)
    g = np.zeros((nt, ntr))
    for f0, c, amp in ((30.0, 1600.0, 1.0), (60.0, 1700.0, 0.6)):
        for r, xr in enumerate(x):
            tau = t - 0.05 - xr / c
            g[:, r] += amp * np.exp(-(tau * f0 * 2.0) ** 2) * np.cos(2 * np.pi * f0 * tau)
    g += 1e-3 * rng.standard_normal(g.shape)
    return g.astype(np.float32), x, fs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("MFDM_REF_ROOT", "/root/reference"))
    args = ap.parse_args()
    spec = importlib.util.spec_from_file_location("ref_test", os.path.join(args.reference, "tools",
                                                                         "test.py"))
    ref = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref)
    g, x, fs = synthetic_gather()
    c_min, c_max, dc = 1400.0, 1900.0, 5.0
    _, _, amp = ref.dispersion_imaging(g.astype(np.float64), x, fs, c_min, c_max, dc)
    cs = np.linspace(1500.0 * (1 + 1e-8), 1800.0 * (1 - 1e-8), 64)
    modes = np.stack([ref.omega_from_c(cs, 1500.0, 1000.0, 3200.0, 1800.0, 2000.0, 100.0, mode=m)
                      for m in range(3)])
    np.savez_compressed(os.path.join(HERE, "dispersion_small.npz"), gather=g, offsets=x, fs=fs,
                        c_min=c_min, c_max=c_max, dc=dc, amplitude=amp, mode_c=cs, mode_omega=modes)
    print("amplitude", amp.shape, float(amp.max()), "modes", modes.shape)


if __name__ == "__main__":
    main()
