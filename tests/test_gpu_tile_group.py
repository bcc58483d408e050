"""Segment height, the tile autotuner and groups of models on a B200.

The segment height only regroups cells into blocks: every cell runs the same
arithmetic, except that a cell may fall in a segment that takes the general
(boundary-capable) body under one height and the interior body under another,
which the compiler may contract into FMAs differently. Results under different
heights therefore agree to FP32 rounding (relative L2 <= 1e-6 here). A group
runs each model's own launches, so every model in a group must match the same
model stepped alone bit for bit.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

modelgen = importlib.import_module("marineseis-fdm-2d_b200.modelgen")


@pytest.fixture(scope="module")
def lib(mfdm):
    mfdm.build()
    mfdm.load_library()
    return mfdm


def run(lib, model, nt, seg=None, tune=False):
    with lib.Solver.from_model(model) as s:
        if seg is not None:
            s.set_tile(seg)
        if tune:
            s.autotune()
        s.set_shot(0, reset=True)
        s.step(nt)
        return s.records(), {n: s.field(n) for n in lib.FIELDS}, s.info()


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("case", ["curv_small", "cpml_curv_small"])
def test_segment_heights_agree(lib, cases, case):
    model = getattr(cases, case)()
    rec0, f0, info0 = run(lib, model, 150)
    assert info0["seg_rows"] == 8  # the default below 6 M cells per launch
    for seg in (4, 12, 24, 48, 128):
        rec, f, info = run(lib, model, 150, seg=seg)
        assert info["seg_rows"] == seg
        for q in rec0:
            assert rel_l2(rec[q], rec0[q]) <= 1e-6, (seg, q)
        for n in f0:
            assert rel_l2(f[n], f0[n]) <= 1e-6, (seg, n)


def test_set_tile_rejects_bad_heights(lib, cases):
    with lib.Solver.from_model(cases.flat_small()) as s:
        for bad in (-4, 2, 6, 132):
            with pytest.raises(lib.MfdmError):
                s.set_tile(bad)
        s.set_tile(0)
        assert s.info()["seg_rows"] == 8


def test_autotune_picks_a_candidate_and_leaves_rest(lib, cases):
    model = cases.curv_small()
    with lib.Solver.from_model(model) as s:
        s.set_shot(0, reset=True)
        s.step(10)
        seg = s.autotune()
        assert seg in (8, 12, 16, 24, 32, 48)
        assert s.info()["blocks_per_sm"] in (2, 3, 4)
        info = s.info()
        assert info["seg_rows"] == seg and info["step"] == 0 and info["nsamples"] == 0
        for n in lib.FIELDS:
            assert not np.any(s.field(n)), n
        # cached: a second handle of the same shape gets the same height
        with lib.Solver.from_model(model) as s2:
            assert s2.autotune() == seg
        s.step(150)
        rec = s.records()
    rec0, _, _ = run(lib, model, 150)
    for q in rec0:
        assert rel_l2(rec[q], rec0[q]) <= 1e-6, q


def test_group_matches_models_alone(lib, cases):
    models = [cases.flat_small(), cases.curv_small(), cases.cpml_curv_small(),
              modelgen.layered(200, 120, seed=11, nt=100)]
    tiles = [0, 8, 16, 48]
    nt = 70  # two captured 32-step replays and six single steps (one before, to start odd)
    alone = []
    for m, seg in zip(models, tiles):
        with lib.Solver.from_model(m) as s:
            s.set_tile(seg)
            s.set_shot(0, reset=True)
            s.step(nt)
            alone.append((s.records(), {n: s.field(n) for n in lib.FIELDS}))
    solvers = [lib.Solver.from_model(m) for m in models]
    try:
        for s, seg in zip(solvers, tiles):
            s.set_tile(seg)
            s.set_shot(0, reset=True)
        with lib.Group(solvers) as g:
            g.step(1)
            g.step(nt - 1)
            for s in solvers:
                assert s.info()["step"] == nt
            for k, s in enumerate(solvers):
                rec = s.records()
                for q in rec:
                    assert np.array_equal(rec[q], alone[k][0][q]), (k, q)
                for n in lib.FIELDS:
                    assert np.array_equal(s.field(n), alone[k][1][n]), (k, n)
            # a model stepped on its own falls out of step with the group
            solvers[0].step(1)
            with pytest.raises(lib.MfdmError):
                g.step(2)
    finally:
        for s in solvers:
            s.close()


def test_group_with_a_batch_and_timing(lib, cases):
    model = cases.curv_small()
    shots = [(70, 44, 25.0, 5.0), (30, 20, 12.5, 3.0)]
    other = cases.flat_small()
    with lib.Batch.from_model(model, shots) as b, lib.Solver.from_model(other) as s:
        s.set_shot(0, reset=True)
        with lib.Group([b, s]) as g:
            ms = g.time_steps(64)
            assert ms > 0.0
        got = [b.records(shot=k) for k in range(2)] + [s.records()]
    with lib.Batch.from_model(model, shots) as b2:
        b2.step(64)
        ref = [b2.records(shot=k) for k in range(2)]
    ref.append(run(lib, other, 64)[0])
    for k in range(3):
        for q in ref[k]:
            assert np.array_equal(got[k][q], ref[k][q]), (k, q)
    with pytest.raises(lib.MfdmError):
        lib.Group([])


@pytest.mark.parametrize("case", ["curv_small", "cpml_curv_small"])
def test_stage_builds_agree(lib, cases, case):
    """The stage builds (TMA rings at 2 and 3 blocks per SM, shared-memory tiles)
    compute the same stencil on the same staged values; they may contract FMAs
    differently, so they agree to FP32 rounding."""
    model = getattr(cases, case)()
    out = {}
    for blocks in (2, 3, 4):
        with lib.Solver.from_model(model) as s:
            s.set_blocks_per_sm(blocks)
            s.set_tile(8)
            assert s.info()["blocks_per_sm"] == blocks
            s.set_shot(0, reset=True)
            s.step(150)
            out[blocks] = (s.records(), {n: s.field(n) for n in lib.FIELDS})
    for b in (3, 4):
        for q in out[2][0]:
            assert rel_l2(out[b][0][q], out[2][0][q]) <= 1e-6, (b, q)
        for n in lib.FIELDS:
            assert rel_l2(out[b][1][n], out[2][1][n]) <= 1e-6, (b, n)
    with lib.Solver.from_model(model) as s:
        with pytest.raises(lib.MfdmError):
            s.set_blocks_per_sm(5)
        s.set_blocks_per_sm(0)
        assert s.info()["blocks_per_sm"] == 3  # the default build


def test_per_kernel_timing_steps_like_step(lib, cases):
    """mfdm_time_steps with per-kernel events launches the steps one by one
    (outside the captured graph, in chunks of 256): the same state as
    mfdm_step, and the five kernel intervals tile each step's interval."""
    model = cases.curv_small()
    nt = 300
    rec0, f0, _ = run(lib, model, nt)
    with lib.Solver.from_model(model) as s:
        s.set_shot(0, reset=True)
        total, kms = s.time_steps(nt, per_kernel=True)
        assert s.info()["step"] == nt
        assert total > 0.0 and len(kms) == 5 and all(k > 0.0 for k in kms)
        assert abs(sum(kms) - total) <= 1e-3 * total + 1e-3
        rec = s.records()
        for q in rec0:
            assert np.array_equal(rec[q], rec0[q]), q
        for n in lib.FIELDS:
            assert np.array_equal(s.field(n), f0[n]), n
