"""Solid only (calc_type 0) on a B200: with a free surface (boundary_type 2, the
reference's PmlFs::SolidOnly) and with CFS-PML on all four sides
(boundary_type 1, Cpml::SolidOnly).

The reference build's records (solid vz on row 3; row 30 with four-side PML)
and final snapshots of two seeded models per boundary type are the golden
fixtures (tests/golden/solid_*.npz, cpml_solid_*.npz, pinned to the FP32
oracle by tests/test_oracle.py); the CUDA path must match them and the
oracle's final fields to a relative L2 of 1e-5.
"""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SOLID = ("solid_flat_small", "solid_curv_small", "cpml_solid_flat_small", "cpml_solid_curv_small")


@pytest.fixture(scope="module")
def lib(mfdm):
    mfdm.build()
    mfdm.load_library()
    return mfdm


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def run(lib, model, nt, shot=0):
    with lib.SolidSolver.from_model(model) as s:
        s.set_shot(shot, reset=True)
        s.step(nt)
        return s.records(), {n: s.field(n) for n in ("solid_vx", "solid_vz", "solid_sx",
                                                     "solid_sz", "solid_sxz")}


@pytest.mark.parametrize("name", SOLID)
def test_solid_only_matches_reference_build(lib, cases, name):
    model = cases.CASES[name][0]()
    d = np.load(cases.fixture_path(name))
    rec, f = run(lib, model, int(d["nt"]))
    assert rec["svz"].shape == d["svz"].shape
    assert rel(rec["svz"], d["svz"]) <= 1e-5
    for comp in ("vx", "vz"):
        assert rel(f["solid_" + comp], d["snap_solid_" + comp]) <= 1e-5, comp


@pytest.mark.parametrize("name", SOLID)
def test_solid_only_fields_match_oracle(lib, oracle, cases, name):
    model = cases.CASES[name][0]()
    nt = 300
    ref = oracle.forward_solid(model, nt, oracle.record_gap(model.dt), 32, final_fields=True)
    rec, f = run(lib, model, nt)
    assert rel(rec["svz"], ref["svz"]) <= 1e-5
    for q, n in enumerate(("solid_vx", "solid_vz", "solid_sx", "solid_sz", "solid_sxz")):
        assert rel(f[n], ref["solid"][q]) <= 1e-5, n


def test_graph_loop_matches_single_steps(lib, cases):
    model = cases.solid_curv_small()
    a, _ = run(lib, model, 70)
    with lib.SolidSolver.from_model(model) as s:
        s.set_shot(0, reset=True)
        for _ in range(70):
            s.step(1)
        b = s.records()
    assert np.array_equal(a["svz"], b["svz"])


def test_cli_writes_the_solid_only_tree(lib, cases, modelgen, tmp_path):
    model = cases.solid_flat_small()
    model.nt, model.snapshot = 120, 50
    j = modelgen.write_model(model, str(tmp_path / "model"))
    out = tmp_path / "out"
    r = subprocess.run([lib.CLI_PATH, j, str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    shot = out / "0"
    assert sorted(os.listdir(shot / "record")) == ["solid_vz.bin"]
    assert sorted(os.listdir(shot / "snapshot")) == ["solid"]
    rec, f = run(lib, model, 120)
    got = np.fromfile(shot / "record" / "solid_vz.bin", dtype="<f4").reshape(rec["svz"].shape)
    assert np.array_equal(got, rec["svz"])
    for it in (0, 50, 100):
        for comp in ("vx", "vz"):
            p = shot / "snapshot" / "solid" / comp / f"{comp}_{it:06d}.bin"
            assert os.path.getsize(p) == model.nz * model.nx * 4
    last = np.fromfile(shot / "snapshot" / "solid" / "vz" / "vz_000100.bin", dtype="<f4")
    _, f101 = run(lib, model, 101)
    assert np.array_equal(last.reshape(model.nz, model.nx), f101["solid_vz"])


def test_cli_runs_four_side_cpml_solid(lib, cases, modelgen, tmp_path):
    """calc_type 0 with boundary_type 1 through the drop-in command line: the
    record file holds solid vz on row 30 (src/main.cu:303-311)."""
    model = cases.cpml_solid_curv_small()
    model.nt, model.snapshot = 150, 100
    j = modelgen.write_model(model, str(tmp_path / "model"))
    out = tmp_path / "out"
    r = subprocess.run([lib.CLI_PATH, j, str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    rec, f = run(lib, model, 150)
    got = np.fromfile(out / "0" / "record" / "solid_vz.bin", dtype="<f4").reshape(rec["svz"].shape)
    assert np.array_equal(got, rec["svz"])
    assert rec["svz"].shape == (75, model.nx) and np.abs(rec["svz"]).max() > 0
    # the last sample is taken after step it = 148, i.e. row 30 of the state after 149 steps
    _, f149 = run(lib, model, 149)
    assert np.array_equal(rec["svz"][-1], f149["solid_vz"][30])


def test_solid_only_rejects_bad_input(lib, cases):
    model = cases.solid_flat_small()
    with lib.SolidSolver.from_model(model) as s:
        with pytest.raises(lib.MfdmError):
            s.set_shot(3)
        with pytest.raises(lib.MfdmError):
            s.field("fluid_p")
    bad = cases.solid_flat_small()
    bad.npd = 60
    with pytest.raises(lib.MfdmError):
        lib.SolidSolver.from_model(bad)
