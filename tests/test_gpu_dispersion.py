"""Phase-shift dispersion imaging on a B200 (mfdm_dispersion_image, the
reference's tools/test.py:50-98): against the reference's own output on a
seeded gather (golden vectors), and on the CUDA path's records of a 100 m
water layer over an elastic half-space, where the image's ridge must follow
the analytic fundamental guided mode (tools/test.py:101-140, `omega_from_c`)."""
import importlib
import os

import numpy as np
import pytest

from oracle import dispersion

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "dispersion_small.npz")


@pytest.fixture(scope="module")
def lib(mfdm):
    mfdm.build()
    mfdm.load_library()
    return mfdm


def test_gpu_image_matches_reference_vectors(lib):
    d = np.load(GOLDEN)
    f, v, a = lib.dispersion_image(d["gather"], d["offsets"], float(d["fs"]), float(d["c_min"]),
                                   float(d["c_max"]), float(d["dc"]))
    assert a.shape == d["amplitude"].shape
    assert np.max(np.abs(a - d["amplitude"])) <= 1e-6
    assert np.allclose(v, dispersion.velocities(float(d["c_min"]), float(d["c_max"]), float(d["dc"])))


def test_gpu_image_rejects_bad_input(lib):
    g = np.zeros((64, 4), np.float32)
    with pytest.raises(lib.MfdmError):
        lib.dispersion_image(g, np.arange(4.0), 1000.0, 1800.0, 1500.0, 1.0)
    with pytest.raises(ValueError):
        lib.dispersion_image(g, np.arange(3.0), 1000.0, 1500.0, 1800.0, 1.0)


def test_guided_mode_of_a_water_layer(lib):
    """100 m of water (vp 1500, rho 1000) over vp 3200, vs 1800, rho 2000 (the
    reference's analysis parameters), flat seafloor, 20 Hz source 50 m below
    the surface, 6000 steps of 0.4 ms: the solid vz record on the seafloor,
    imaged at 1450..1850 m/s, peaks within 1 % of the first guided mode above
    its cutoff (branch `mode=1` of omega_from_c; branch 0 has positive
    frequencies only below 2.8 Hz here) from 12 to 35 Hz (measured with the
    oracle: within 0.35 %)."""
    mg = importlib.import_module("marineseis-fdm-2d_b200.modelgen")
    m = mg.make_model(1000, 24, 83, h=5.0, npd=20, fpeak=20.0, dt=4e-4, nt=6000, vp_f=1500.0,
                      rho_f=1000.0, vp=3200.0, vs=1800.0, rho=2000.0, src_x=[60], src_z=[13])
    with lib.Solver.from_model(m) as s:
        s.set_shot(0, reset=True)
        s.step(m.nt)
        rec = s.records()
        gap = s.info()["gap"]
    fs = 1.0 / (gap * m.dt)
    cols = np.arange(100, 900)
    x = (cols - 60) * m.h
    g = rec["svz"][:, cols]
    f, v, a = lib.dispersion_image(g, x, fs, 1450.0, 1850.0, 2.0)
    fo, vo, ao = dispersion.dispersion_image(g, x, fs, 1450.0, 1850.0, 2.0)
    assert np.max(np.abs(a - ao)) <= 1e-6
    cs = np.linspace(1500.001, 1799.999, 20000)
    w = dispersion.omega_from_c(cs, 1500.0, 1000.0, 3200.0, 1800.0, 2000.0, 100.0, 1)
    ok = np.isfinite(w) & (w > 0)
    fr, cr = w[ok] / (2 * np.pi), cs[ok]
    order = np.argsort(fr)
    assert fr.min() < 12.0 and fr.max() > 35.0
    for fq in (12.0, 15.0, 20.0, 25.0, 30.0, 35.0):
        k = int(round(fq / (fs / g.shape[0])))
        theory = float(np.interp(f[k], fr[order], cr[order]))
        peak = float(v[np.argmax(a[k])])
        assert abs(peak - theory) <= 0.01 * theory, (f[k], peak, theory)
