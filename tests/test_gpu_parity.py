"""Parity of the CUDA path (libmfdm.so through its C ABI) on a B200.

* against records of the reference's own CUDA build (tests/golden, produced by
  oracle/_ref/main_debug on a B200) for every golden case, full length, up to
  the 1200 x 800 (6000 steps) and 4096 x 2048 (1500 steps) models; past 1500
  steps also against the FP32 noise floor measured between two builds of the
  reference that differ only in FMA contraction, and against the FP64 oracle;
* against the CPU oracle (FP32 and FP64) on whole wavefields;
* through size-independent properties at the 4096 x 2048 size (linearity,
  oracle agreement over a bounded number of steps);
* the drop-in CLI's output tree and the multi-shot and error behaviour;
* the four-side CFS-PML variant (boundary_type 1, Cpml::FluidSolid) on its
  own reference-build fixtures.

Tolerance: relative L2 <= 1e-5 in FP32 (per record trace set / per field).
"""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5
ALL_CASES = ["flat_small", "curv_small", "shallow_src", "flat_400x400", "curvilinear_1200x800",
             "curvilinear_4096x2048", "cpml_flat_small", "cpml_curv_small"]
# Past 1500 steps the distance to the reference build may also be at most this
# multiple of the distance between the reference build and the same sources
# built with FMA contraction off (both FP32, same algorithm, same order), when
# that is the larger bound. Measured (1200 x 800, 6000 steps): this path
# 3.6-4.0e-6 from the reference build, the two reference builds 6.5-8.6e-7
# apart, the reference build 3.3-4.6e-6 from the FP64 oracle.
NOISE_MULT = 8.0


@pytest.fixture(scope="module")
def lib(mfdm):
    mfdm.build()
    mfdm.load_library()
    return mfdm


def run_solver(mfdm, model, nt, fields=True):
    with mfdm.Solver.from_model(model) as s:
        s.set_shot(0, reset=True)
        s.step(nt)
        rec = s.records()
        out = {n: s.field(n) for n in mfdm.FIELDS} if fields else None
        info = s.info()
    return rec, out, info


PREFIX_STEPS = 1500


@pytest.mark.parametrize("name", ALL_CASES)
def test_records_match_reference_build(lib, cases, name):
    """<= 1e-5 against the reference build over the whole record and the final
    snapshot (whole, or every k-th row and column at the large sizes); the
    first 1500 steps are also checked on their own. For the long runs the
    fixture holds the distance between two reference builds that differ only in
    FMA contraction (the FP32 rounding-noise floor) and the FP64 oracle's
    records: the CUDA path must stay within max(1e-5, NOISE_MULT x floor) of
    the reference build and no further from the FP64 records than
    max(1e-5, 1.5 x the reference build's own distance to them)."""
    build, stride, keep = cases.CASES[name]
    step = cases.snapshot_step(keep)
    model = build()
    g = np.load(cases.fixture_path(name))
    nt = int(g["nt"])
    rec, fields, info = run_solver(lib, model, nt, fields=bool(step))
    assert info["nsamples"] == g["svx"].shape[0]
    gap = info["gap"]
    npre = -(-min(nt, PREFIX_STEPS) // gap)
    report = {}
    for k in ("svx", "svz", "fp"):
        e = rel_l2(rec[k][:npre, ::stride], g[k][:npre])
        report[k + "_prefix"] = e
        assert e <= TOL, (name, k, "prefix", e)
    if step:
        for key, arr in (("snap_solid_vx", fields["solid_vx"]), ("snap_solid_vz", fields["solid_vz"]),
                         ("snap_fluid_vx", fields["fluid_vx"]), ("snap_fluid_vz", fields["fluid_vz"])):
            e = rel_l2(arr[::step, ::step], g[key])
            report[key] = e
            assert e <= TOL, (name, key, e)
    if nt > PREFIX_STEPS:
        for k in ("svx", "svz", "fp"):
            e_ref = rel_l2(rec[k][:, ::stride], g[k])
            report[k + "_full"] = e_ref
            assert e_ref <= TOL, (name, k, "full record", e_ref)
            if "nofma_rel_l2_" + k in g:
                floor = float(g["nofma_rel_l2_" + k])
                report[k + "_noise_floor"] = floor
                assert e_ref <= max(TOL, NOISE_MULT * floor), (name, k, e_ref, floor)
            if "fp64_" + k in g:
                s64 = int(g["fp64_stride"]) if "fp64_stride" in g else stride
                ours64 = rel_l2(rec[k][:, ::s64], g["fp64_" + k])
                ref64 = rel_l2(g[k][:, ::s64 // stride], g["fp64_" + k])
                report[k + "_fp64"] = ours64
                report[k + "_ref_fp64"] = ref64
                assert ours64 <= max(TOL, 1.5 * ref64), (name, k, ours64, ref64)
    print(name, {k: f"{v:.3e}" for k, v in report.items()})


@pytest.mark.parametrize("name", ["flat_small", "curv_small", "shallow_src", "cpml_flat_small",
                                  "cpml_curv_small"])
def test_all_fields_match_oracle(lib, oracle, cases, name):
    model = cases.CASES[name][0]()
    nt = model.nt
    rec, fields, _ = run_solver(lib, model, nt)
    for prec in (32, 64):
        ref = oracle.forward(model, nt, oracle.record_gap(model.dt), prec, final_fields=True)
        for q, n in enumerate(("fluid_vx", "fluid_vz", "fluid_p")):
            assert rel_l2(fields[n], ref["fluid"][q]) <= TOL, (prec, n)
        for q, n in enumerate(("solid_vx", "solid_vz", "solid_sx", "solid_sz", "solid_sxz")):
            assert rel_l2(fields[n], ref["solid"][q]) <= TOL, (prec, n)
        for k in ("svx", "svz", "fp"):
            assert rel_l2(rec[k], ref[k]) <= TOL, (prec, k)


def test_update_rk4_matches_graph_loop(lib, cases):
    """The single-step seam and the captured time loop run the same kernels."""
    model = cases.curv_small()
    n = 70  # two graph replays (32 steps each) plus direct launches
    with lib.Solver.from_model(model) as s:
        s.set_shot(0, reset=True)
        s.step(n)
        ra, fa = s.records(), s.field("solid_sxz")
        s.set_shot(0, reset=True)
        for it in range(n):
            s.update_rk4(it)
        s.synchronize()
        rb, fb = s.records(), s.field("solid_sxz")
    for k in ra:
        assert np.array_equal(ra[k], rb[k])
    assert np.array_equal(fa, fb)


def test_cli_output_tree_and_bytes(lib, cases, modelgen, tmp_path):
    model = cases.curv_small()
    model.nt, model.snapshot = 250, 100
    j = modelgen.write_model(model, str(tmp_path / "model"))
    out = tmp_path / "out"
    (out / "stale").mkdir(parents=True)
    r = subprocess.run([lib.CLI_PATH, j, str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert not (out / "stale").exists()  # out_root is cleared first (src/main.cu:83)
    shot = out / "0"
    gap = 3
    ns = -(-250 // gap)
    for f in ("solid_vx", "solid_vz", "fluid_p"):
        assert os.path.getsize(shot / "record" / f"{f}.bin") == ns * model.nx * 4
    for it in (0, 100, 200):
        for medium, rows in (("solid", model.nz_s), ("fluid", model.nz_f)):
            for comp in ("vx", "vz"):
                p = shot / "snapshot" / medium / comp / f"{comp}_{it:06d}.bin"
                assert os.path.getsize(p) == rows * model.nx * 4, p
    assert not (shot / "snapshot" / "solid" / "vx" / "vx_000249.bin").exists()
    rec, _, _ = run_solver(lib, model, 250, fields=False)
    got = np.fromfile(shot / "record" / "fluid_p.bin", dtype="<f4").reshape(ns, model.nx)
    assert np.array_equal(got, rec["fp"])
    # in-process entry point writes the same bytes
    out2 = tmp_path / "out2"
    lib.run_cli(j, str(out2))
    for f in ("solid_vx", "solid_vz", "fluid_p"):
        assert (out2 / "0" / "record" / f"{f}.bin").read_bytes() == (shot / "record" / f"{f}.bin").read_bytes()


def test_multishot_keeps_wavefield_between_shots(lib, cases, modelgen, tmp_path):
    """The reference never clears the fields between shots (src/main.cu:94-136)."""
    model = cases.flat_small()
    model.nt = 120
    model.src_x, model.src_z = [40, 80], [40, 30]
    j = modelgen.write_model(model, str(tmp_path / "model"))
    out = tmp_path / "out"
    r = subprocess.run([lib.CLI_PATH, j, str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    with lib.Solver.from_model(model) as s:
        s.set_shot(0, reset=True)
        s.step(120)
        s.set_shot(1, reset=False)
        s.step(120)
        carried = s.records()
        s.set_shot(1, reset=True)
        s.step(120)
        fresh = s.records()
    got = np.fromfile(out / "1" / "record" / "solid_vz.bin", dtype="<f4").reshape(carried["svz"].shape)
    assert np.array_equal(got, carried["svz"])
    assert not np.array_equal(carried["svz"], fresh["svz"])


def test_nonfinite_is_reported(lib, modelgen):
    model = modelgen.make_model(64, 24, 32, npd=6, dt=4e-3, nt=400, src_x=[32], src_z=[16])
    with lib.Solver.from_model(model) as s:
        s.set_shot(0, reset=True)
        with pytest.raises(lib.MfdmError) as ei:
            s.step(400)
        assert ei.value.code == -5


def test_linearity_at_full_size(lib, modelgen):
    """One step is linear in the state: doubling every field doubles the result
    (scaling by 2 is exact in FP32, so the comparison is tight)."""
    model = modelgen.curvilinear_4096x2048(nt=10)
    rng = np.random.default_rng(11)
    init = {}
    for n in lib.FIELDS:
        rows = model.nz_f if n.startswith("fluid") else model.nz_s
        init[n] = (rng.standard_normal((rows, model.nx)) * 1e-3).astype(np.float32)
    res = []
    with lib.Solver.from_model(model) as s:
        for scale in (1.0, 2.0):
            s.set_shot(0, reset=True)
            for n, v in init.items():
                s.set_field(n, v * np.float32(scale))
            for it in range(1000, 1006):  # Ricker is zero after 2 * 1.2 / fpeak
                s.update_rk4(it)
            s.synchronize()
            res.append({n: s.field(n) for n in lib.FIELDS})
    for n in lib.FIELDS:
        assert rel_l2(res[1][n], 2.0 * res[0][n]) <= 1e-12, n


def test_full_size_against_oracle(lib, oracle, modelgen):
    """4096 x 2048 curvilinear model, first 40 steps, every field against the FP32 oracle."""
    model = modelgen.curvilinear_4096x2048(nt=40)
    rec, fields, info = run_solver(lib, model, 40)
    assert info["cells"] == 4096 * 2049
    ref = oracle.forward(model, 40, oracle.record_gap(model.dt), 32, final_fields=True)
    for q, n in enumerate(("fluid_vx", "fluid_vz", "fluid_p")):
        assert rel_l2(fields[n], ref["fluid"][q]) <= TOL, n
    for q, n in enumerate(("solid_vx", "solid_vz", "solid_sx", "solid_sz", "solid_sxz")):
        assert rel_l2(fields[n], ref["solid"][q]) <= TOL, n


def test_largest_size_against_oracle(lib, oracle, modelgen):
    """The 8192 x 4096 rough-seafloor model of the batched adjoint (33.6 M cells,
    von Karman seafloor, flat side pads), first 20 steps of shot 0, every field
    against the FP32 oracle: the index arithmetic and launch shapes at the
    largest configured size."""
    model = modelgen.rough_seafloor(8192, 4096, nt=20)
    rec, fields, info = run_solver(lib, model, 20)
    assert info["cells"] == model.cells
    ref = oracle.forward(model, 20, oracle.record_gap(model.dt), 32, final_fields=True)
    for q, n in enumerate(("fluid_vx", "fluid_vz", "fluid_p")):
        assert rel_l2(fields[n], ref["fluid"][q]) <= TOL, n
    for q, n in enumerate(("solid_vx", "solid_vz", "solid_sx", "solid_sz", "solid_sxz")):
        assert rel_l2(fields[n], ref["solid"][q]) <= TOL, n
