"""CPU oracle of the phase-shift dispersion image and of the analytic guided-mode
curves of a fluid layer over an elastic half-space (test infrastructure only).

Restates the reference's tools/test.py:
* `dispersion_image` follows `dispersion_imaging` (tools/test.py:50-98): real
  FFT of every trace over time, phase spectrum conj(S)/|S| (0 where |S| = 0),
  normalised stack over the traces of exp(-i w x / c) for every frequency bin
  and test velocity numpy.arange(c_min, c_max + dc/2, dc); FP64 throughout.
* `omega_from_c` follows `omega_from_c` (tools/test.py:101-140): the
  dispersion relation of the modes of a fluid layer of thickness H (speed
  alpha_w, density rho_w) over a half-space (alpha, beta, rho), defined for
  alpha_w < c < min(alpha, beta).
Pinned to the reference's own functions by the golden vectors in
tests/golden/dispersion_small.npz (tests/golden/make_dispersion_golden.py).
"""
from __future__ import annotations

import numpy as np


def velocities(c_min: float, c_max: float, dc: float) -> np.ndarray:
    return np.arange(c_min, c_max + dc / 2.0, dc)


def dispersion_image(gather, offsets, fs: float, c_min: float, c_max: float, dc: float):
    """(frequencies [nf], velocities [nv], amplitude [nf][nv]) of a gather [nt][ntr]."""
    g = np.asarray(gather, dtype=np.float64)
    x = np.asarray(offsets, dtype=np.float64)
    nt, ntr = g.shape
    spec = np.fft.rfft(g, axis=0)
    freqs = np.fft.rfftfreq(nt, d=1.0 / fs)
    mag = np.abs(spec)
    phase = np.zeros_like(spec)
    np.divide(spec.conj(), mag, out=phase, where=mag > 0)
    vel = velocities(c_min, c_max, dc)
    w = 2.0 * np.pi * freqs
    amp = np.empty((freqs.size, vel.size))
    for k in range(freqs.size):
        shift = np.exp(-1j * w[k] * x[:, None] / vel[None, :])
        amp[k] = np.abs(phase[k] @ shift) / ntr
    return freqs, vel, amp


def omega_from_c(c, alpha_w, rho_w, alpha, beta, rho, thickness, mode=0):
    """Angular frequency of mode `mode` at phase velocity c (NaN outside
    alpha_w < c < min(alpha, beta))."""
    c = np.atleast_1d(np.asarray(c, dtype=np.float64))
    out = np.full(c.shape, np.nan)
    ok = np.isfinite(c) & (c > alpha_w) & (c < alpha) & (c < beta)
    cv = c[ok]
    a = cv ** 2 / alpha_w ** 2 - 1.0
    b = 1.0 - cv ** 2 / alpha ** 2
    q = 1.0 - cv ** 2 / beta ** 2
    d = 1.0 / alpha_w ** 2 - 1.0 / cv ** 2
    ratio = rho * beta ** 4 * np.sqrt(a) / (rho_w * cv ** 4 * np.sqrt(b))
    bracket = 4.0 * np.sqrt(q) * np.sqrt(b) - (cv ** 2 / beta ** 2 - 2.0) ** 2
    out[ok] = (np.arctan(ratio * bracket) + mode * np.pi) / (thickness * np.sqrt(d))
    return out
