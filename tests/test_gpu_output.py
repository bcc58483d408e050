"""The output path on a B200: asynchronously drained snapshots, the opt-in
fluid pressure snapshots and the batched command line with one output tree per
shot.

Every drained snapshot must hold exactly the state the solver has after that
step (the staging copy runs on the compute stream before the next step), and
every shot of the batched command line must write the records of the same shot
run alone from rest.
"""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NT, SNAP = 90, 10


@pytest.fixture(scope="module")
def lib(mfdm):
    mfdm.build()
    mfdm.load_library()
    return mfdm


def snap(path, rows, nx):
    return np.fromfile(path, dtype="<f4").reshape(rows, nx)


def solver_states(lib, model, shot, steps_wanted):
    """Fields of `shot` (from rest) after steps it+1 for every it in steps_wanted, and the records."""
    out = {}
    with lib.Solver.from_model(model) as s:
        s.set_shot(shot, reset=True)
        done = 0
        for it in sorted(steps_wanted):
            s.step(it + 1 - done)
            done = it + 1
            out[it] = {n: s.field(n) for n in ("fluid_vx", "fluid_vz", "fluid_p", "solid_vx", "solid_vz")}
        s.step(model.nt - done)
        return out, s.records()


def check_tree(lib, model, shot_dir, shot, pressure):
    its = list(range(0, model.nt, SNAP))
    states, rec = solver_states(lib, model, shot, its)
    for it in its:
        for medium, rows in (("solid", model.nz_s), ("fluid", model.nz_f)):
            comps = ("vx", "vz", "p") if (medium == "fluid" and pressure) else ("vx", "vz")
            for comp in comps:
                p = shot_dir / "snapshot" / medium / comp / f"{comp}_{it:06d}.bin"
                assert np.array_equal(snap(p, rows, model.nx), states[it][f"{medium}_{comp}"]), p
    assert not (shot_dir / "snapshot" / "fluid" / "p").exists() or pressure
    ns = rec["fp"].shape[0]
    for f, k in (("solid_vx", "svx"), ("solid_vz", "svz"), ("fluid_p", "fp")):
        got = np.fromfile(shot_dir / "record" / f"{f}.bin", dtype="<f4").reshape(ns, model.nx)
        assert np.array_equal(got, rec[k]), (f, shot)


def test_drained_snapshots_hold_the_state_of_their_step(lib, cases, modelgen, tmp_path):
    model = cases.curv_small()
    model.nt, model.snapshot = NT, SNAP  # a snapshot every 10 steps: both staging slots cycle
    j = modelgen.write_model(model, str(tmp_path / "model"))
    out = tmp_path / "out"
    r = subprocess.run([lib.CLI_PATH, j, str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    check_tree(lib, model, out / "0", 0, pressure=False)


def test_pressure_snapshots_on_request(lib, cases, modelgen, tmp_path):
    model = cases.flat_small()
    model.nt, model.snapshot = NT, SNAP
    j = modelgen.write_model(model, str(tmp_path / "model"))
    out = tmp_path / "out"
    env = dict(os.environ, MFDM_SNAPSHOT_PRESSURE="1")
    r = subprocess.run([lib.CLI_PATH, j, str(out)], capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr
    check_tree(lib, model, out / "0", 0, pressure=True)


def test_batched_cli_writes_each_shot_as_run_alone(lib, cases, modelgen, tmp_path):
    model = cases.curv_small()
    model.nt, model.snapshot = NT, SNAP
    model.src_x, model.src_z = [70, 30, 100], [44, 20, 40]
    j = modelgen.write_model(model, str(tmp_path / "model"))
    out = tmp_path / "out"
    env = dict(os.environ, MFDM_BATCH="1", MFDM_SNAPSHOT_PRESSURE="1")
    r = subprocess.run([lib.CLI_PATH, j, str(out)], capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr
    for shot in range(3):
        check_tree(lib, model, out / str(shot), shot, pressure=True)
    # the in-process entry point writes the same bytes
    out2 = tmp_path / "out2"
    lib.run_cli_batch(j, str(out2))
    for shot in range(3):
        for f in ("solid_vx", "solid_vz", "fluid_p"):
            a = (out / str(shot) / "record" / f"{f}.bin").read_bytes()
            assert (out2 / str(shot) / "record" / f"{f}.bin").read_bytes() == a
