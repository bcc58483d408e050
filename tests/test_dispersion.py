"""Phase-shift dispersion imaging: the CPU oracle against golden vectors of the
reference's own `dispersion_imaging` and `omega_from_c` (tools/test.py:50-140),
evaluated by tests/golden/make_dispersion_golden.py on a seeded gather."""
import os

import numpy as np

from oracle import dispersion

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "dispersion_small.npz")


def test_oracle_image_matches_reference_vectors():
    d = np.load(GOLDEN)
    f, v, a = dispersion.dispersion_image(d["gather"].astype(np.float64), d["offsets"], float(d["fs"]),
                                          float(d["c_min"]), float(d["c_max"]), float(d["dc"]))
    assert a.shape == d["amplitude"].shape == (129, 101)
    assert np.max(np.abs(a - d["amplitude"])) <= 1e-12
    assert v[0] == 1400.0 and v[-1] == 1900.0 and f[1] == float(d["fs"]) / 256


def test_oracle_mode_curves_match_reference_vectors():
    d = np.load(GOLDEN)
    for m in range(3):
        w = dispersion.omega_from_c(d["mode_c"], 1500.0, 1000.0, 3200.0, 1800.0, 2000.0, 100.0, m)
        ref = d["mode_omega"][m]
        assert np.array_equal(np.isnan(w), np.isnan(ref))
        ok = ~np.isnan(ref)
        assert np.allclose(w[ok], ref[ok], rtol=1e-13, atol=0.0)
    # outside alpha_w < c < min(alpha, beta): NaN
    assert np.isnan(dispersion.omega_from_c([1400.0, 1900.0], 1500.0, 1000.0, 3200.0, 1800.0,
                                            2000.0, 100.0)).all()


def test_image_of_a_plane_wave_peaks_at_its_velocity():
    """A non-dispersive train at 1650 m/s images at 1650 m/s in every band with signal."""
    fs, nt, ntr, c0 = 1000.0, 512, 64, 1650.0
    x = 20.0 + 5.0 * np.arange(ntr)
    t = np.arange(nt) / fs
    g = np.stack([np.exp(-((t - 0.05 - xr / c0) * 60.0) ** 2) for xr in x], axis=1)
    f, v, a = dispersion.dispersion_image(g, x, fs, 1500.0, 1800.0, 2.0)
    band = (f >= 10.0) & (f <= 60.0)
    assert np.all(np.abs(v[np.argmax(a[band], axis=1)] - c0) <= 2.0)
