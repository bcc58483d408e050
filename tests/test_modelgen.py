"""The seeded model generator: metric identities and the on-disk format."""
import json
import os

import numpy as np


def test_flat_metric_is_cartesian(modelgen):
    m = modelgen.flat_400x400(nt=10)
    assert (m.nx, m.nz_f, m.nz_s, m.nz) == (400, 204, 197, 400)
    h = m.h
    assert np.allclose(m.metric["J"], h * h)
    assert np.allclose(m.metric["xi_x"], 1 / h) and np.allclose(m.metric["ze_z"], 1 / h)
    assert not m.metric["xi_z"].any() and not m.metric["ze_x"].any()
    assert m.beta0 == 5.0 and m.thickness == 95.0
    assert (m.src_x[0], m.src_z[0]) == (200, 193)


def test_curvilinear_metric_identities(modelgen):
    m = modelgen.curvilinear(300, 200, zeta0=100, nt=10)
    J, zx, zz = m.metric["J"], m.metric["ze_x"], m.metric["ze_z"]
    z = m.metric["z"]
    # J = h z_zeta and ze_x = -z_xi / J against centred differences of z
    dz_dze = np.gradient(z, axis=0)
    dz_dxi = np.gradient(z, axis=1)
    inner = (slice(2, -2), slice(2, -2))
    assert np.allclose(J[inner], m.h * dz_dze[inner], rtol=2e-3)
    assert np.allclose(zx[inner], (-dz_dxi / J)[inner], rtol=2e-3, atol=1e-4)
    assert np.allclose(zz, m.h / J)
    # seafloor on row zeta0 follows 40 sin(2 pi x / 600) about the flat depth
    x = m.h * np.arange(m.nx)
    assert np.allclose(z[100], m.h * 97 + 40 * np.sin(2 * np.pi * x / 600))
    # the bottom PML band is flat: constant row spacing h in every column
    b = m.nz - 4 - m.npd
    assert np.allclose(J[b:], m.h * m.h)


def test_perturbations_seeded_and_bounded(modelgen):
    a = modelgen.curvilinear(200, 120, zeta0=60, nt=10, seed=1)
    b = modelgen.curvilinear(200, 120, zeta0=60, nt=10, seed=1)
    c = modelgen.curvilinear(200, 120, zeta0=60, nt=10, seed=2)
    assert np.array_equal(a.solid["C11"], b.solid["C11"])
    assert not np.array_equal(a.solid["C11"], c.solid["C11"])
    rho = a.solid["rho"]
    assert rho.min() >= 2000 * 0.95 - 1e-9 and rho.max() <= 2000 * 1.05 + 1e-9


def test_write_model_reference_layout(modelgen, tmp_path):
    m = modelgen.make_model(40, 16, 20, npd=4, nt=10)
    j = modelgen.write_model(m, str(tmp_path / "case"), name="case")
    cfg = json.load(open(j))
    assert set(cfg) == {"base", "grid", "PML"}
    assert cfg["grid"]["calc_type"] == 1 and cfg["grid"]["boundary_type"] == 2
    assert set(cfg["grid"]["jacob"]) == {"J", "xi_x", "xi_z", "ze_x", "ze_z"}
    c11 = np.fromfile(cfg["grid"]["solid"]["C11"], dtype="<f4")
    assert c11.size == 40 * 20
    jac = np.fromfile(cfg["grid"]["jacob"]["J"], dtype="<f4")
    assert jac.size == 40 * (16 + 20 - 1)
    rel = modelgen.write_model(m, str(tmp_path / "rel"), relative_to=str(tmp_path))
    cfg = json.load(open(rel))
    assert not os.path.isabs(cfg["grid"]["fluid"]["K"])
