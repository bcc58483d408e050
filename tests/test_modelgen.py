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
    pad = m.pad
    assert pad == m.npd + 3
    # J = h z_zeta and ze_x = -z_xi / J against centred differences of z, away
    # from the two columns where the flat pads meet the physical domain
    dz_dze = np.gradient(z, axis=0)
    dz_dxi = np.gradient(z, axis=1)
    cols = np.r_[2:pad - 1, pad + 2:m.nx - pad - 2, m.nx - pad + 2:m.nx - 2]
    assert np.allclose(J[2:-2][:, cols], m.h * dz_dze[2:-2][:, cols], rtol=2e-3)
    assert np.allclose(zx[2:-2][:, cols], (-dz_dxi / J)[2:-2][:, cols], rtol=2e-3, atol=1e-4)
    assert np.allclose(zz, m.h / J)
    # seafloor on row zeta0 follows 40 sin(2 pi x / 600), x the physical
    # coordinate h (xi - pad), about the flat depth inside the physical domain
    x = m.h * (np.arange(m.nx) - pad)
    phys = slice(pad, m.nx - pad)
    assert np.allclose(z[100, phys], m.h * 97 + 40 * np.sin(2 * np.pi * x[phys] / 600))
    # the bottom PML band is flat: constant row spacing h in every column
    b = m.nz - 4 - m.npd
    assert np.allclose(J[b:], m.h * m.h)


def test_side_pads_are_flat(modelgen):
    """The outer npd + 3 columns hold every grid line at the end column's depth
    (model_FANDS_PANDF_double_cos_padmove.py:199-203)."""
    m = modelgen.curvilinear_1200x800(nt=10)
    z, pad = m.metric["z"], m.pad
    assert np.array_equal(z[:, :pad], np.repeat(z[:, pad:pad + 1], pad, axis=1))
    assert np.array_equal(z[:, -pad:], np.repeat(z[:, -pad - 1:-pad], pad, axis=1))
    assert not m.metric["ze_x"][:, :pad].any() and not m.metric["ze_x"][:, -pad:].any()
    assert np.allclose(m.metric["J"][:, :pad], m.h * m.h)
    # the physical domain does undulate
    assert np.ptp(z[m.nz_f - 1, pad:-pad]) > 70.0


def test_cpml_top_band_is_flat(modelgen):
    """With CFS-PML on all four sides the blend starts below the top band
    (row npd + 3), so that band has the same thickness in every column."""
    m = modelgen.make_model(128, 52, 64, npd=12, nt=10, amp=20.0, wavelength=300.0,
                            boundary_type=1)
    top = m.npd + 3
    assert np.allclose(m.metric["J"][:top + 1], m.h * m.h)
    assert not m.metric["ze_x"][:top + 1].any()
    assert m.metric["ze_x"][m.nz_f - 1].any()


def test_pad_txt_written_and_read(modelgen, tmp_path):
    m = modelgen.curvilinear(200, 120, zeta0=60, nt=10)
    j = modelgen.write_model(m, str(tmp_path / "case"), name="case")
    pad = modelgen.read_pad(os.path.join(os.path.dirname(j), "pad.txt"))
    assert pad["pad_flat"] == pad["shift"] == m.npd + 3
    assert pad["nx_phys"] == m.nx - 2 * (m.npd + 3)
    assert pad["phys0"] == m.npd + 3 and pad["phys1"] == m.nx - m.npd - 4
    assert pad["nz_fluid_full"] == m.nz_f and pad["nz_solid_full"] == m.nz_s
    assert pad["nz_fluid_phys"] == m.nz_f - 3 and pad["src_z_offset"] == 3


def test_von_karman_profile(modelgen):
    g, dg = modelgen.von_karman_profile(4000, 5.0, seed=5)
    g2, _ = modelgen.von_karman_profile(4000, 5.0, seed=5)
    g3, _ = modelgen.von_karman_profile(4000, 5.0, seed=6)
    assert np.array_equal(g, g2) and not np.array_equal(g, g3)
    assert abs(np.sqrt(np.mean(g ** 2)) - 20.0) < 1e-9 and abs(g.mean()) < 1e-9
    # the derivative along xi agrees with centred differences of the band-limited profile
    assert np.allclose(np.gradient(g)[1:-1], dg[1:-1], atol=0.05 * np.abs(dg).max())
    # correlation: neighbouring samples 5 m apart are almost equal, 1 km apart nearly independent
    c = lambda lag: np.corrcoef(g[:-lag], g[lag:])[0, 1]
    assert c(1) > 0.95 and abs(c(200)) < 0.3


def test_rough_seafloor_model(modelgen):
    m = modelgen.rough_seafloor(nx=1024, nz=512, nt=10, nshots=4)
    pad = m.pad
    sea = m.metric["z"][m.nz_f - 1] - m.h * (m.nz_f - 1 - 3)
    assert abs(np.sqrt(np.mean(sea[pad:-pad] ** 2)) - 20.0) < 2.0
    assert np.all(sea[:pad] == sea[pad]) and np.all(sea[-pad:] == sea[-pad - 1])
    assert len(m.src_x) == 4 and all(pad < x < m.nx - pad for x in m.src_x)
    assert m.fpeak == 10.0 and np.all(m.metric["J"] > 0)


def test_adjoint_pair(modelgen):
    true, init = modelgen.adjoint_pair(400, 200, nt=10)
    vs = lambda m: np.sqrt(m.solid["C55"] / m.solid["rho"])
    vp = lambda m: np.sqrt(m.solid["C11"] / m.solid["rho"])
    base = modelgen.curvilinear(400, 200, nt=10, seed=1)
    ratio = vs(true) / vs(base)
    assert np.isclose(ratio.max(), 1.10, atol=1e-3)  # +10 % at the centre
    iz, ix = np.unravel_index(np.argmax(ratio), ratio.shape)
    z = true.metric["z"][true.nz_f - 1:]
    assert ix == 200 and abs(z[iz, ix] - z[0, ix] - 150.0) <= true.h
    assert np.allclose(vp(true), vp(base))  # vp and rho unchanged
    assert np.array_equal(true.metric["J"], init.metric["J"])
    assert np.array_equal(true.fluid["K"], init.fluid["K"])
    # the initial model is smooth: the anomaly is largely gone
    assert (vs(init) / vs(base)).max() < 1.05


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
