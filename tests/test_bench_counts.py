"""The byte counts bench.py divides by (no GPU needed).

The roofline of the RK4 step counts 16 state floats (stage inputs, U^n, the
accumulator and the outputs over the four stages) and 4 coefficient reads per
field and cell: 464 B a solid cell, 288 B a fluid cell, and 256 B per PML strip
cell and direction for the four ADE memory fields. The batched form reads the
coefficients once for all shots of a segment.
"""
import importlib
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
bench = importlib.import_module("bench")
modelgen = importlib.import_module("marineseis-fdm-2d_b200.modelgen")


def small():
    return modelgen.make_model(96, 40, 44, npd=10, dt=2e-4, nt=10, src_x=[48], src_z=[20])


def test_algorithmic_bytes_per_cell_rule():
    m = small()
    strips = 2 * m.npd * (m.nz_f - 3) + 2 * m.npd * (m.nz_s - 3) + m.npd * (m.nx - 6)
    expect = m.nx * m.nz_f * 288 + m.nx * m.nz_s * 464 + strips * 256
    assert bench.algorithmic_bytes(m) == expect


def test_batched_bytes_share_only_the_coefficients():
    m = small()
    one = bench.batched_bytes(m, 1)
    assert one == bench.algorithmic_bytes(m)
    coef = (m.nx * m.nz_f * 4 * 6 + m.nx * m.nz_s * 4 * 9) * 4
    for n in (2, 8, 64):
        assert bench.batched_bytes(m, n) == n * (one - coef) + coef


def test_both_arms_print_the_same_config():
    class Args:
        workload = "flat_400x400"
    m = bench.WORKLOADS["flat_400x400"]()
    cfg = bench.bench_config(Args(), m, 1)
    assert cfg["workload"] == "flat_400x400"
    assert cfg["cells"] == m.nx * (m.nz_f + m.nz_s)
    assert bench.bench_config(Args(), m, 1) == cfg
