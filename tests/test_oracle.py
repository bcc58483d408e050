"""The CPU oracle against records of the reference's own CUDA build.

The fixtures in tests/golden were produced on a B200 by oracle/_ref/main_debug,
the unmodified reference sources compiled for sm_100a (tests/golden/make_golden.py).
FP32 tolerance: relative L2 <= 1e-5 per record, the bound the port is held to.
"""
import numpy as np
import pytest

from conftest import rel_l2

TOL = 1e-5


def _check_case(oracle, cases, name, nsteps=None, precision=32):
    build, stride, keep = cases.CASES[name]
    k = cases.snapshot_step(keep)
    model = build()
    g = np.load(cases.fixture_path(name))
    nt = int(g["nt"]) if nsteps is None else nsteps
    gap = oracle.record_gap(model.dt)
    out = oracle.forward(model, nt, gap, precision, final_fields=bool(k) and nsteps is None)
    ns = out["svx"].shape[0]
    errs = {r: rel_l2(out[r][:, ::stride], g[r][:ns]) for r in ("svx", "svz", "fp")}
    if k and nsteps is None:
        errs["snap_solid_vx"] = rel_l2(out["solid"][0][::k, ::k], g["snap_solid_vx"])
        errs["snap_solid_vz"] = rel_l2(out["solid"][1][::k, ::k], g["snap_solid_vz"])
        errs["snap_fluid_vx"] = rel_l2(out["fluid"][0][::k, ::k], g["snap_fluid_vx"])
        errs["snap_fluid_vz"] = rel_l2(out["fluid"][1][::k, ::k], g["snap_fluid_vz"])
    return errs, out, g


@pytest.mark.parametrize("name", ["flat_small", "curv_small", "shallow_src", "cpml_flat_small",
                                  "cpml_curv_small"])
def test_oracle_matches_reference_small(oracle, cases, name):
    errs, _, g = _check_case(oracle, cases, name)
    assert float(g["run_to_run_rel_l2"]) == 0.0
    for k, e in errs.items():
        assert e <= TOL, (name, k, e)


def test_oracle_matches_reference_flat_400x400(oracle, cases):
    errs, out, _ = _check_case(oracle, cases, "flat_400x400")
    assert out["svx"].shape == (1000, 400)  # gap 2 at dt = 0.5 ms
    for k, e in errs.items():
        assert e <= TOL, (k, e)


def test_oracle_matches_reference_curvilinear_prefix(oracle, cases):
    # 1500 of the 6000 steps keep the CPU suite short; the full run is a GPU test.
    errs, out, _ = _check_case(oracle, cases, "curvilinear_1200x800", nsteps=1500)
    assert out["svx"].shape[0] == 500  # gap 3 at dt = 0.4 ms
    for k, e in errs.items():
        assert e <= TOL, (k, e)


def test_fp32_against_fp64_oracle(oracle, cases):
    model = cases.curv_small()
    gap = oracle.record_gap(model.dt)
    a = oracle.forward(model, model.nt, gap, 32)
    b = oracle.forward(model, model.nt, gap, 64)
    for k in ("svx", "svz", "fp"):
        assert rel_l2(a[k], b[k]) <= TOL


def test_planted_mistake_is_detected(oracle, cases):
    """The comparison is sensitive: moving the source one cell breaks the match."""
    model = cases.flat_small()
    model.src_x = [model.src_x[0] + 1]
    g = np.load(cases.fixture_path("flat_small"))
    out = oracle.forward(model, int(g["nt"]), oracle.record_gap(model.dt), 32)
    assert rel_l2(out["fp"], g["fp"]) > 1e-3


def test_record_gap_rounding(oracle):
    # (int)(1e-3 / float(dt) + 0.5) (src/main.cu:92): 0.4 ms gives 3 through float rounding.
    assert oracle.record_gap(5e-4) == 2
    assert oracle.record_gap(4e-4) == 3
    assert oracle.record_gap(1e-4) == 10


@pytest.mark.parametrize("name", ["solid_flat_small", "solid_curv_small", "cpml_solid_flat_small",
                                  "cpml_solid_curv_small"])
def test_solid_only_oracle_matches_reference(oracle, cases, name):
    """Solid only (calc_type 0): PmlFs::SolidOnly (boundary_type 2) and
    Cpml::SolidOnly (boundary_type 1), the FP32 restatement against the
    reference build's solid vz record (row 3 / row 30) and its final solid
    snapshot."""
    model = cases.CASES[name][0]()
    d = np.load(cases.fixture_path(name))
    r = oracle.forward_solid(model, int(d["nt"]), oracle.record_gap(model.dt), 32,
                             final_fields=True)
    assert np.linalg.norm(r["svz"] - d["svz"]) <= 2e-6 * np.linalg.norm(d["svz"])
    for q, comp in ((0, "vx"), (1, "vz")):
        ref = d["snap_solid_" + comp]
        assert np.linalg.norm(r["solid"][q] - ref) <= 5e-6 * np.linalg.norm(ref), comp
