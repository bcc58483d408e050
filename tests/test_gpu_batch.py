"""Batched shots (mfdm_open_batch) on a B200.

A batch steps several shots of one model with one launch per RK stage. Every
shot must come out bit for bit as the same shot run alone through the
single-shot path (which tests/test_gpu_parity.py holds to the reference build
and the oracle): same source cell, same Ricker frequency and the PML alpha0 /
beta0 that go with it, starting from rest.
"""
import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (src_x, src_z, fpeak, beta0): different sources, frequencies and PML beta0,
# and one shot without a source (its wavefield stays at rest).
SHOTS = [(70, 44, 25.0, 5.0), (30, 20, 12.5, 3.0), (100, 40, 40.0, 1.5), (-1, 0, 20.0, 2.0)]


@pytest.fixture(scope="module")
def lib(mfdm):
    mfdm.build()
    mfdm.load_library()
    return mfdm


def single_shot(lib, model, shot, nt):
    m = copy.deepcopy(model)
    x, z, f, b = shot
    m.src_x, m.src_z = ([x], [z]) if x >= 0 else ([], [])
    m.fpeak, m.beta0 = f, b
    with lib.Solver.from_model(m) as s:
        s.set_shot(0, reset=True)
        s.step(nt)
        return s.records(), {n: s.field(n) for n in lib.FIELDS}


@pytest.mark.parametrize("case", ["curv_small", "cpml_curv_small"])
def test_batch_matches_single_shots(lib, cases, case):
    model = getattr(cases, case)()
    nt = 200
    with lib.Batch.from_model(model, SHOTS) as b:
        assert b.info()["nshots"] == len(SHOTS)
        b.step(nt)
        got = [(b.records(shot=k), {n: b.field(n, shot=k) for n in lib.FIELDS})
               for k in range(len(SHOTS))]
    for k, shot in enumerate(SHOTS):
        rec, fields = single_shot(lib, model, shot, nt)
        for q in ("svx", "svz", "fp"):
            assert np.array_equal(got[k][0][q], rec[q]), (k, q)
        for n in lib.FIELDS:
            assert np.array_equal(got[k][1][n], fields[n]), (k, n)
    # the shot without a source stays at rest; the others do not
    assert not np.any(got[3][0]["fp"])
    assert all(np.any(got[k][0]["fp"]) for k in range(3))


def test_batch_reset_repeats_and_rejects_bad_input(lib, cases):
    model = cases.flat_small()
    with lib.Batch.from_model(model, SHOTS[:2]) as b:
        b.step(70)  # two graph replays (32 steps) plus single steps
        first = b.records(shot=1)
        b.reset()
        b.step(70)
        again = b.records(shot=1)
        for q in first:
            assert np.array_equal(first[q], again[q])
        with pytest.raises(lib.MfdmError):
            b.set_shot(0)
        with pytest.raises(lib.MfdmError):
            b.records(shot=2)
    with pytest.raises(lib.MfdmError):
        lib.Batch.from_model(model, [(60, 40, 0.0, 5.0)])  # fpeak must be > 0
    with pytest.raises(lib.MfdmError):
        lib.Batch.from_model(model, [(60, 500, 25.0, 5.0)])  # source below the fluid
