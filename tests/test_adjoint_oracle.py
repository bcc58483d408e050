"""The FP64 adjoint oracle (oracle/adjoint.py) against the oracle itself.

The reference has no adjoint, so the oracle's adjoint is pinned by the two
properties that define it: its assembled operators reproduce the oracle's own
stage RHS and filter, and its gradients agree with central finite differences
of the oracle's FP64 misfit (relative error <= 1e-6 at eps = 1e-4, where the
O(eps^2) truncation is about 1e-8).
"""
import importlib

import numpy as np
import pytest

modelgen = importlib.import_module("marineseis-fdm-2d_b200.modelgen")

NSTEPS = 120


def tiny_model(boundary_type=2):
    m = modelgen.make_model(48, 24, 28, npd=8, fpeak=30.0, dt=5e-4, nt=NSTEPS, src_x=[24],
                            src_z=[17], amp=10.0, wavelength=150.0, perturb=0.05, seed=3)
    m.boundary_type = boundary_type
    return m


def records(pyoracle, model, nsteps, gap):
    out = pyoracle.forward(model, nsteps, gap, precision=64, round_inputs=False)
    return np.stack([out["svx"], out["svz"], out["fp"]], axis=1)


@pytest.fixture(scope="module", params=[2, 1], ids=["free_surface", "cpml"])
def setup(request, oracle):
    from oracle import adjoint as A
    model = tiny_model(request.param)
    adj = A.OracleAdjoint(model)
    p = A.params_of(model)
    # observed data: +5% vs in a Gaussian blob below the seafloor
    q = {k: v.copy() for k, v in p.items()}
    xx, zz = np.meshgrid(np.arange(model.nx), np.arange(model.nz_s))
    q["vs"] = q["vs"] * (1 + 0.05 * np.exp(-((xx - 24) ** 2 + (zz - 8) ** 2) / 20.0))
    obs = records(oracle, A.with_params(model, q), NSTEPS, adj.gap)
    yield A, adj, model, p, obs
    adj.close()


def test_assembled_operators_reproduce_the_oracle(setup):
    A, adj, model, p, obs = setup
    rng = np.random.default_rng(0)
    x = rng.standard_normal(adj.lay.n)
    for d in (0, 1):
        ref = adj.h.rhs(d, x)
        assert np.linalg.norm(adj.L[d] @ x - ref) <= 1e-13 * np.linalg.norm(ref)
    ref = adj.h.filter(x)
    assert np.linalg.norm(adj.F @ x - ref) <= 1e-13 * np.linalg.norm(ref)


def test_forward_with_saved_stages_matches_the_oracle(setup, oracle):
    A, adj, model, p, obs = setup
    rec, ys = adj.forward(NSTEPS)
    assert len(ys) == NSTEPS and ys[0].shape == (4, adj.lay.n)
    assert np.array_equal(rec, records(oracle, model, NSTEPS, adj.gap))
    assert np.any(rec[:, 2])


def test_gradient_matches_finite_differences(setup, oracle):
    A, adj, model, p, obs = setup
    rec, ys = adj.forward(NSTEPS)
    _, res = A.misfit(rec, obs)
    gp = A.chain_rule(adj.gradient(NSTEPS, res, ys), p)
    rng = np.random.default_rng(4)
    eps = 1e-4
    for name in ("vp", "vs", "rho", "vp_f", "rho_f"):
        dlt = rng.standard_normal(p[name].shape) * p[name] * 1e-2
        dj = float(np.sum(gp[name] * dlt))
        jp = A.misfit(records(oracle, A.with_params(model, {**p, name: p[name] + eps * dlt}),
                              NSTEPS, adj.gap), obs)[0]
        jm = A.misfit(records(oracle, A.with_params(model, {**p, name: p[name] - eps * dlt}),
                              NSTEPS, adj.gap), obs)[0]
        fd = (jp - jm) / (2 * eps)
        assert dj != 0.0, name
        assert abs(fd - dj) <= 1e-6 * abs(dj), (name, fd, dj)
