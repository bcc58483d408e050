"""Adjoint-state gradients (mfdm_adjoint_forward / _backward) on a B200.

The reference has no adjoint; the library's gradients are held to
* the FP64 adjoint oracle (oracle/adjoint.py, itself pinned to finite
  differences of the FP64 oracle) for the same fixed receiver residuals:
  relative L2 <= 1e-3 per coefficient array (the FP32 forward trajectory and
  FP32 transposed products against FP64);
* central finite differences of the library's own FP32 misfit along seeded
  smooth random directions: agreement <= 1e-3 at a relative step of 1e-3
  (a white-noise direction mostly cancels in the misfit, and FP32 rounding of
  the records then dominates the difference).
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

modelgen = importlib.import_module("marineseis-fdm-2d_b200.modelgen")
grads = importlib.import_module("marineseis-fdm-2d_b200.gradients")

NSTEPS = 120


def tiny_model(boundary_type=2):
    # no flat side pads: on 48 columns they would leave 26 physical ones
    return modelgen.make_model(48, 24, 28, npd=8, fpeak=30.0, dt=5e-4, nt=NSTEPS, src_x=[24],
                               src_z=[17], amp=10.0, wavelength=150.0, perturb=0.05, seed=3,
                               boundary_type=boundary_type, flat_sides=False)


@pytest.fixture(scope="module")
def lib(mfdm):
    mfdm.build()
    mfdm.load_library()
    return mfdm


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("bdy", [2, 1], ids=["free_surface", "cpml"])
def test_gradient_matches_fp64_adjoint_oracle(lib, oracle, bdy):
    from oracle import adjoint as A
    model = tiny_model(bdy)
    gap = oracle.record_gap(model.dt)
    ns = -(-NSTEPS // gap)
    rng = np.random.default_rng(7)
    res = rng.standard_normal((ns, 3, model.nx)).astype(np.float32)
    res[:, :, :3] = 0.0
    res[:, :, -3:] = 0.0
    adj = A.OracleAdjoint(model, round_inputs=True)
    try:
        _, ys = adj.forward(NSTEPS)
        ref = adj.gradient(NSTEPS, res.astype(np.float64), ys)
    finally:
        adj.close()
    with lib.Solver.from_model(model) as s:
        s.set_shot(0, reset=True)
        rec = s.adjoint_forward(NSTEPS, ckpt_every=25)
        assert rec["fp"].shape == (ns, model.nx) and np.any(rec["fp"])
        g = s.adjoint_backward({"svx": res[:, 0], "svz": res[:, 1], "fp": res[:, 2]})
        assert s.info()["step"] == 0
    names = {"K": "K", "rcp_rho_f": "rf", "C11": "C11", "C13": "C13", "C33": "C33",
             "C55": "C55", "rcp_rho_s": "rs"}
    for k, ko in names.items():
        assert np.any(ref[ko]), k
        assert rel(g[k], ref[ko]) <= 1e-3, (k, rel(g[k], ref[ko]))


def test_checkpoint_interval_does_not_change_the_gradient(lib):
    model = tiny_model()
    rng = np.random.default_rng(3)
    out = []
    with lib.Solver.from_model(model) as s:
        s.set_shot(0, reset=True)
        ns = -(-NSTEPS // s.info()["gap"])
        res = {k: rng.standard_normal((ns, model.nx)).astype(np.float32) for k in ("svx", "svz", "fp")}
        for every in (1, 7, 50, NSTEPS):
            s.adjoint_forward(NSTEPS, ckpt_every=every)
            out.append(s.adjoint_backward(res))
    for g in out[1:]:
        for k in g:
            assert np.array_equal(g[k], out[0][k]), k


def test_kept_segments_give_the_same_gradient(lib):
    """Stage inputs kept from the forward pass (mfdm_adjoint_set_memory) instead of
    recomputed from checkpoints: the same kernels on the same inputs, bit for bit."""
    model = tiny_model()
    rng = np.random.default_rng(11)
    out = []
    with lib.Solver.from_model(model) as s:
        s.set_shot(0, reset=True)
        ns = -(-NSTEPS // s.info()["gap"])
        res = {k: rng.standard_normal((ns, model.nx)).astype(np.float32) for k in ("svx", "svz", "fp")}
        info = s.info()
        # bytes of one segment's stage inputs, at least (4 states per step, 25 steps,
        # the 8 main fields; the ADE strips make a set a little larger)
        seg_bytes = 25 * 4 * 4 * 8 * (info["nz_f"] + info["nz_s"]) * info["pitch"]
        recs = []
        for nb in (0, 2 * seg_bytes, 1 << 40, 0):  # none, one or two, all five, none
            s.adjoint_memory(nb)
            recs.append(s.adjoint_forward(NSTEPS, ckpt_every=25))
            out.append(s.adjoint_backward(res))
    for g in out[1:]:
        for k in g:
            assert np.array_equal(g[k], out[0][k]), k
    # kept steps run their stages in place in the keep buffer: the same records
    for r in recs[1:]:
        for k in r:
            assert np.array_equal(r[k], recs[0][k]), k
    with lib.Solver.from_model(model) as s:
        with pytest.raises(lib.MfdmError):
            s.adjoint_memory(-1)


def test_two_checkpoint_levels_give_the_same_gradient(lib):
    """Inner checkpoints re-run each segment once more; the stage inputs are the
    same values, so the gradient is the same bit for bit."""
    model = tiny_model()
    rng = np.random.default_rng(12)
    out = []
    with lib.Solver.from_model(model) as s:
        s.set_shot(0, reset=True)
        ns = -(-NSTEPS // s.info()["gap"])
        res = {k: rng.standard_normal((ns, model.nx)).astype(np.float32) for k in ("svx", "svz", "fp")}
        for inner in (0, 7, 1, 0):
            s.adjoint_inner(inner)
            s.adjoint_forward(NSTEPS, ckpt_every=40)
            out.append(s.adjoint_backward(res))
        with pytest.raises(lib.MfdmError):
            s.adjoint_inner(-1)
    for g in out[1:]:
        for k in g:
            assert np.array_equal(g[k], out[0][k]), k


def test_gradient_matches_finite_differences(lib):
    model = tiny_model()
    p = grads.params_of(model)
    q = {k: v.copy() for k, v in p.items()}
    xx, zz = np.meshgrid(np.arange(model.nx), np.arange(model.nz_s))
    q["vs"] = q["vs"] * (1 + 0.05 * np.exp(-((xx - 24) ** 2 + (zz - 8) ** 2) / 20.0))

    def records(s, prm):
        s.load_model(grads.with_params(model, prm))
        s.set_shot(0, reset=True)
        s.step(NSTEPS)
        r = s.records()
        return np.stack([r["svx"], r["svz"], r["fp"]], axis=1).astype(np.float64)

    with lib.Solver.from_model(model) as s:
        obs = records(s, q)
        s.load_model(grads.with_params(model, p))
        s.set_shot(0, reset=True)
        rec = s.adjoint_forward(NSTEPS, ckpt_every=30)
        r = np.stack([rec["svx"], rec["svz"], rec["fp"]], axis=1).astype(np.float64) - obs
        g = grads.chain_rule(s.adjoint_backward({"svx": r[:, 0], "svz": r[:, 1], "fp": r[:, 2]}), p)
        rng = np.random.default_rng(4)
        for name in ("vp", "vs", "rho", "vp_f", "rho_f"):
            # a smooth seeded direction (Gaussian-correlated, 4 cells), 1e-3 of the parameter
            dlt = modelgen._correlated_field(rng, p[name].shape, 4.0) * p[name] * 1e-3
            dj = float(np.sum(g[name] * dlt))
            jp = 0.5 * np.sum((records(s, {**p, name: p[name] + dlt}) - obs) ** 2)
            jm = 0.5 * np.sum((records(s, {**p, name: p[name] - dlt}) - obs) ** 2)
            fd = (jp - jm) / 2.0
            assert abs(fd - dj) <= 1e-3 * abs(dj), (name, fd, dj)


def test_adjoint_rejects_misuse(lib, cases):
    model = tiny_model()
    with lib.Solver.from_model(model) as s:
        with pytest.raises(lib.MfdmError):
            s.adjoint_backward({})  # no forward run
        s.set_shot(0, reset=True)
        s.adjoint_forward(20, ckpt_every=10)
        s.step(1)
        with pytest.raises(lib.MfdmError):
            s.adjoint_backward({})  # a step after the forward run
        with pytest.raises(lib.MfdmError):
            s.adjoint_forward(0, 10)
    with lib.Batch.from_model(cases.flat_small(), [(60, 40, 25.0, 5.0)]) as b:
        with pytest.raises(lib.MfdmError):
            b.adjoint_forward(10)


def test_shot_gradients_sum_over_shots(lib):
    shots_mod = importlib.import_module("marineseis-fdm-2d_b200.shots")
    model = tiny_model()
    model.src_x, model.src_z = [20, 30], [17, 15]
    rng = np.random.default_rng(5)
    with lib.Solver.from_model(model) as s:
        ns = -(-NSTEPS // s.info()["gap"])
    obs = {k: {q: rng.standard_normal((ns, model.nx)).astype(np.float32) * 1e-9
               for q in ("svx", "svz", "fp")} for k in range(2)}
    j, g = shots_mod.shot_gradients_on_gpu(model, [0, 1], obs, ckpt_every=40)
    parts = [shots_mod.shot_gradients_on_gpu(model, [k], obs, ckpt_every=40) for k in range(2)]
    assert j == pytest.approx(parts[0][0] + parts[1][0], rel=1e-12)
    # float32 sums on the device: shot 0 + shot 1 in that order, exactly
    assert g.is_cuda and g.dtype == torch_float32()
    assert np.array_equal(g.cpu().numpy(), (parts[0][1] + parts[1][1]).cpu().numpy())
    # and the device sum equals the host gradients rounded to float32
    with lib.Solver.from_model(model) as s:
        s.set_shot(0, reset=True)
        rec = s.adjoint_forward(NSTEPS, 40)
        host = s.adjoint_backward({k: (rec[k] - obs[0][k]).astype(np.float32) for k in rec})
    flat = np.concatenate([host[k].astype(np.float32).ravel() for k in shots_mod.GRAD_KEYS])
    assert np.array_equal(parts[0][1].cpu().numpy(), flat)
    # the single-process gradient_shots returns the same sums as [rows][nx] views
    shapes = {k: host[k].shape for k in shots_mod.GRAD_KEYS}
    j2, g2 = shots_mod.gradient_shots(model, obs, shapes)
    assert j2 == pytest.approx(j, rel=1e-7)
    for k in shots_mod.GRAD_KEYS:
        assert g2[k].shape == shapes[k]
    assert np.array_equal(np.concatenate([g2[k].cpu().numpy().ravel() for k in shots_mod.GRAD_KEYS]),
                          g.cpu().numpy())


def torch_float32():
    import torch
    return torch.float32


def test_autograd_function_returns_the_adjoint_gradient(lib):
    torch = pytest.importorskip("torch")
    model = tiny_model()
    p = grads.params_of(model)
    t = {k: torch.tensor(v, dtype=torch.float64, requires_grad=True) for k, v in p.items()}
    with lib.Solver.from_model(model) as s:
        s.set_shot(0, reset=True)
        rec = grads.SeismicRecords.apply(t["vp"], t["vs"], t["rho"], t["vp_f"], t["rho_f"], s,
                                         model, NSTEPS, 40)
        w = torch.linspace(-1.0, 1.0, rec.numel(), dtype=torch.float64).reshape(rec.shape)
        (rec * w).sum().backward()
        # the same through the C ABI directly
        s.load_model(grads.with_params(model, p))
        s.set_shot(0, reset=True)
        s.adjoint_forward(NSTEPS, 40)
        wn = w.numpy().astype(np.float32)
        g = grads.chain_rule(s.adjoint_backward({"svx": wn[:, 0], "svz": wn[:, 1], "fp": wn[:, 2]}), p)
    for k in p:
        assert np.array_equal(t[k].grad.numpy(), g[k]), k
