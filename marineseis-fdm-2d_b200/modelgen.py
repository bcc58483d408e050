"""Seeded synthetic marine models in the reference's on-disk format.

The solver reads a JSON config plus little-endian float32 ``[rows][nx]``
binaries (reference ``json_template.json`` and ``docs/io.md``). This module
builds such models with the conventions of the reference's generator scripts
(``tools/run_models/model_FANDS_PANDF_wavy.py:100-177``,
``tools/run_models/model_ortho_freesurface_scholte.py:93-184``):

* three frozen rows on top, the free surface on global row 3;
* the fluid-solid interface on fluid row ``nz_f - 1`` == solid row 0
  (global row ``nz_f - 1``); the metric arrays cover ``nz_f + nz_s - 1`` rows;
* ``x = h * xi`` (vertical grid columns), so ``xi_x = 1/h``, ``xi_z = 0``,
  ``J = h * z_zeta``, ``ze_x = -z_xi / J``, ``ze_z = h / J``
  (``model_FANDS_PANDF_wavy.py:139-144``), evaluated in FP64 from analytic
  derivatives of the grid map;
* the vertical undulation envelope vanishes inside the bottom PML band, so the
  band has the same thickness in every column (``docs/io.md:65-66``);
* the outer ``npd + 3`` columns on each side (3 frozen + the PML band) are a
  flat pad: every grid line there is held at the value of the physical
  domain's end column, physical ``x = h (xi - pad)``
  (``model_FANDS_PANDF_double_cos_padmove.py:120-130, 199-203``), and
  ``write_model`` writes the pad description ``pad.txt`` beside the JSON
  (``…double_cos_padmove.py:296-310``); with CFS-PML on all four sides the
  blend starts below the top band (row ``npd + 3``), so that band is flat too
  (``…double_cos_padmove.py:111``);
* seafloor shapes: a sinusoid, or a seeded von Kármán random profile
  (``von_karman_profile``);
* ``beta0 = min(vs, vp_fluid) / (0.5 * ppw * h * fpeak)`` and
  ``thickness = (npd - 1) * h`` (``model_FANDS_PANDF_wavy.py:174-177``).

Every array is returned in FP64; ``write_model`` rounds to float32 on disk.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

SOLID_FIELDS = ("C11", "C13", "C33", "C55", "rho")
FLUID_FIELDS = ("K", "rho")
METRIC_FIELDS = ("J", "xi_x", "xi_z", "ze_x", "ze_z")


@dataclass
class Model:
    """A fluid-over-solid model on a curvilinear grid (calc_type 1). boundary_type 2:
    free surface on top, CFS-PML left, right and bottom; 1: CFS-PML on all four
    sides (a top PML band in the fluid instead of the free surface)."""

    nx: int
    nz_f: int
    nz_s: int
    h: float
    fpeak: float
    dt: float
    nt: int
    snapshot: int
    src_x: List[int]
    src_z: List[int]
    npd: int
    npow: int
    thickness: float
    vp_max: float
    rc: float
    beta0: float
    fluid: Dict[str, np.ndarray] = field(default_factory=dict)   # [nz_f][nx]
    solid: Dict[str, np.ndarray] = field(default_factory=dict)   # [nz_s][nx]
    metric: Dict[str, np.ndarray] = field(default_factory=dict)  # [nz_f+nz_s-1][nx]
    boundary_type: int = 2
    pad: int = 0  # flat pad columns on each side (npd + 3; 0: no pad)

    @property
    def nz(self) -> int:
        return self.nz_f + self.nz_s - 1

    @property
    def cells(self) -> int:
        """Cells the reference updates per step (the interface row counts twice)."""
        return self.nx * (self.nz_f + self.nz_s)

    def config(self, paths: Dict[str, str]) -> dict:
        """JSON document in the reference schema (json_template.json:1-50)."""
        return {
            "base": {"fpeak": self.fpeak, "dt": self.dt, "nt": int(self.nt),
                     "snapshot": int(self.snapshot)},
            "grid": {
                "calc_type": 1,
                "boundary_type": int(self.boundary_type),
                "src_pos": {"posx": [int(v) for v in self.src_x],
                            "posz": [int(v) for v in self.src_z]},
                "solid": {"nx": self.nx, "nz": self.nz_s,
                          **{k: paths["solid/" + k] for k in SOLID_FIELDS}},
                "jacob": {k: paths["jacob/" + k] for k in METRIC_FIELDS},
                "fluid": {"nx": self.nx, "nz": self.nz_f,
                          **{k: paths["fluid/" + k] for k in FLUID_FIELDS}},
            },
            "PML": {"npd": self.npd, "thickness": self.thickness, "NPOW": self.npow,
                    "Vp_max": self.vp_max, "Rc": self.rc, "beta0": self.beta0},
        }


@dataclass
class SolidModel:
    """A solid with a free surface on top (calc_type 0, boundary_type 2, the
    reference's PmlFs::SolidOnly): all arrays are [nz][nx], the free surface is
    global row 3, CFS-PML left, right and bottom."""

    nx: int
    nz: int
    h: float
    fpeak: float
    dt: float
    nt: int
    snapshot: int
    src_x: List[int]
    src_z: List[int]
    npd: int
    npow: int
    thickness: float
    vp_max: float
    rc: float
    beta0: float
    solid: Dict[str, np.ndarray] = field(default_factory=dict)   # [nz][nx]
    metric: Dict[str, np.ndarray] = field(default_factory=dict)  # [nz][nx]
    boundary_type: int = 2

    @property
    def cells(self) -> int:
        return self.nx * self.nz

    def config(self, paths: Dict[str, str]) -> dict:
        """JSON document in the reference schema with calc_type 0 (no fluid section)."""
        return {
            "base": {"fpeak": self.fpeak, "dt": self.dt, "nt": int(self.nt),
                     "snapshot": int(self.snapshot)},
            "grid": {
                "calc_type": 0,
                "boundary_type": int(self.boundary_type),
                "src_pos": {"posx": [int(v) for v in self.src_x],
                            "posz": [int(v) for v in self.src_z]},
                "solid": {"nx": self.nx, "nz": self.nz,
                          **{k: paths["solid/" + k] for k in SOLID_FIELDS}},
                "jacob": {k: paths["jacob/" + k] for k in METRIC_FIELDS},
            },
            "PML": {"npd": self.npd, "thickness": self.thickness, "NPOW": self.npow,
                    "Vp_max": self.vp_max, "Rc": self.rc, "beta0": self.beta0},
        }


def write_model(model: Model, directory: str, name: str = "model",
                relative_to: Optional[str] = None) -> str:
    """Writes ``<directory>/<name>.json`` and the float32 binaries; returns the JSON path.

    Paths in the JSON are absolute unless ``relative_to`` is given, in which
    case they are relative to that directory (the reference resolves them
    against the working directory, ``src/elements.cu:161``).
    """
    os.makedirs(directory, exist_ok=True)
    paths = {}
    groups = [("solid", model.solid, SOLID_FIELDS), ("jacob", model.metric, METRIC_FIELDS)]
    if not isinstance(model, SolidModel):
        groups.append(("fluid", model.fluid, FLUID_FIELDS))
    for sub, arrays, names in groups:
        os.makedirs(os.path.join(directory, sub), exist_ok=True)
        for k in names:
            p = os.path.abspath(os.path.join(directory, sub, k + ".bin"))
            np.ascontiguousarray(arrays[k], dtype="<f4").tofile(p)
            paths[sub + "/" + k] = os.path.relpath(p, relative_to) if relative_to else p
    jpath = os.path.join(directory, name + ".json")
    with open(jpath, "w") as f:
        json.dump(model.config(paths), f, indent=2)
        f.write("\n")
    if getattr(model, "pad", 0) > 0:
        with open(os.path.join(directory, "pad.txt"), "w") as f:
            f.write(pad_text(model))
    return jpath


def pad_text(model: Model) -> str:
    """The pad description the reference's generators write beside the model
    (``…double_cos_padmove.py:296-310``): physical extent, shift of the physical
    domain and the padded sizes, one ``key value`` pair per line."""
    pad = model.pad
    rows = [("nx_phys", model.nx - 2 * pad), ("shift", pad), ("pad_flat", pad), ("outer", pad),
            ("npd", model.npd), ("nz_fluid_phys", model.nz_f - 3),
            ("nz_solid_phys", model.nz_s - (model.npd + 3)), ("nz_fluid_full", model.nz_f),
            ("nz_solid_full", model.nz_s), ("src_z_offset", 3), ("phys0", pad),
            ("phys1", model.nx - pad - 1)]
    return "".join(f"{k} {v}\n" for k, v in rows)


def read_pad(path: str) -> Dict[str, int]:
    """Parses a ``pad.txt`` (``tools/compare_sem_scholte.py:59-65`` reads ``pad_flat`` from it)."""
    out = {}
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) == 2:
                out[parts[0]] = int(parts[1])
    return out


def _smootherstep(t: np.ndarray) -> np.ndarray:
    t = np.clip(t, 0.0, 1.0)
    return t * t * t * (t * (6.0 * t - 15.0) + 10.0)


def _dsmootherstep(t: np.ndarray) -> np.ndarray:
    inside = (t > 0.0) & (t < 1.0)
    tc = np.clip(t, 0.0, 1.0)
    return np.where(inside, 30.0 * tc * tc * (tc - 1.0) ** 2, 0.0)


def sinusoid_profile(nx: int, h: float, amp: float, wavelength: float,
                     pad: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    """Seafloor perturbation ``amp sin(2 pi x / wavelength)`` per column with
    physical ``x = h (xi - pad)``, and its derivative along xi (FP64)."""
    x = h * (np.arange(nx, dtype=np.float64) - pad)
    if not amp:
        return np.zeros(nx), np.zeros(nx)
    g = amp * np.sin(2.0 * math.pi * x / wavelength)
    dg = amp * (2.0 * math.pi * h / wavelength) * np.cos(2.0 * math.pi * x / wavelength)
    return g, dg


def von_karman_profile(nx: int, h: float, *, hurst: float = 0.7, rms: float = 20.0,
                       corr: float = 200.0, seed: int = 5,
                       min_wavelength: Optional[float] = None) -> Tuple[np.ndarray, np.ndarray]:
    """Seeded 1-D von Kármán random profile (FP64) with its derivative along xi.

    Power spectrum ``(1 + k^2 a^2)^-(H + 1/2)`` (correlation length ``a``, Hurst
    exponent ``H``; the 1-D von Kármán form), synthesised with random phases on
    a periodic line of at least twice ``nx`` columns so the window does not
    wrap, mean removed and scaled to the given rms. Wavelengths shorter than
    ``min_wavelength`` (default 10 h) are removed with a cosine roll-off from
    1.25 times that wavelength, so the grid resolves every undulation (the
    unfiltered spectrum falls only as k^-2.4 and gives grid-scale slopes above
    1). The derivative is the spectral derivative of the same series, exact at
    the grid columns."""
    rng = np.random.default_rng(seed)
    n = 1 << int(math.ceil(math.log2(2 * nx)))
    k = 2.0 * math.pi * np.fft.rfftfreq(n, d=h)
    amp = (1.0 + (k * corr) ** 2) ** (-(hurst + 0.5) / 2.0)
    amp[0] = 0.0
    kc = 2.0 * math.pi / (min_wavelength if min_wavelength else 10.0 * h)
    k0 = 0.8 * kc
    roll = np.clip((k - k0) / (kc - k0), 0.0, 1.0)
    amp *= 0.5 * (1.0 + np.cos(math.pi * roll))
    spec = amp * (rng.standard_normal(k.size) + 1j * rng.standard_normal(k.size))
    if n % 2 == 0:
        spec[-1] = spec[-1].real
    g = np.fft.irfft(spec, n)[:nx]
    dg = np.fft.irfft(1j * k * spec, n)[:nx] * h
    mean = g.mean()
    scale = rms / np.sqrt(np.mean((g - mean) ** 2))
    return (g - mean) * scale, dg * scale


def _flat_pads(g: np.ndarray, dg: np.ndarray, pad: int) -> Tuple[np.ndarray, np.ndarray]:
    """Holds the outer ``pad`` columns on each side at the physical domain's end
    values (slope 0 there; ``…double_cos_padmove.py:199-203``)."""
    g, dg = g.copy(), dg.copy()
    nx = g.size
    if pad > 0:
        g[:pad], g[nx - pad:] = g[pad], g[nx - pad - 1]
        dg[:pad], dg[nx - pad:] = 0.0, 0.0
    return g, dg


def _grid_metric(nx: int, nz_f: int, nz_s: int, npd: int, h: float,
                 g: np.ndarray, dg: np.ndarray, top: int = 3) -> Dict[str, np.ndarray]:
    """FP64 metric of z(xi, zeta) = h (zeta - 3) + g(xi) u(zeta) v(zeta), g the
    seafloor perturbation per column and dg its derivative along xi.

    u rises 0 -> 1 (smootherstep) between row ``top`` (the free surface, row 3,
    or the inner edge of a top PML band) and the interface row; v falls 1 -> 0
    (cos^2) between the interface row and b = nz - 4 - npd, the last undamped
    row above the bottom band (``model_FANDS_PANDF_double_cos_padmove.py:177-189``).
    """
    nz = nz_f + nz_s - 1
    zeta = np.arange(nz, dtype=np.float64)
    zeta0 = float(nz_f - 1)
    b = float(nz - 4 - npd)
    a = float(top)
    tu = (zeta - a) / (zeta0 - a)
    u, du = _smootherstep(tu), _dsmootherstep(tu) / (zeta0 - a)
    v = np.ones(nz)
    dv = np.zeros(nz)
    if b > zeta0:
        seg = zeta > zeta0
        t = np.clip((zeta[seg] - zeta0) / (b - zeta0), 0.0, 1.0)
        v[seg] = np.cos(0.5 * math.pi * t) ** 2
        dv[seg] = np.where(t < 1.0, -0.5 * math.pi / (b - zeta0) * np.sin(math.pi * t), 0.0)
    w, dw = u * v, du * v + u * dv
    z_xi = dg[None, :] * w[:, None]
    z_ze = h + g[None, :] * dw[:, None]
    if np.any(z_ze <= 0.0):
        raise ValueError("grid folds: z_zeta <= 0")
    J = h * z_ze
    x = h * np.arange(nx, dtype=np.float64)
    return {"J": J, "xi_x": np.full((nz, nx), 1.0 / h), "xi_z": np.zeros((nz, nx)),
            "ze_x": -z_xi / J, "ze_z": h / J,
            "x": np.broadcast_to(x[None, :], (nz, nx)).copy(),
            "z": h * (zeta[:, None] - 3.0) + g[None, :] * w[:, None]}


def _correlated_field(rng: np.random.Generator, shape, corr_cells: float) -> np.ndarray:
    """Zero-mean Gaussian-correlated field scaled to max |value| = 1 (FFT filter)."""
    noise = rng.standard_normal(shape)
    ky = np.fft.fftfreq(shape[0])[:, None]
    kx = np.fft.rfftfreq(shape[1])[None, :]
    kern = np.exp(-2.0 * (math.pi * corr_cells) ** 2 * (kx * kx + ky * ky))
    f = np.fft.irfft2(np.fft.rfft2(noise) * kern, s=shape)
    f -= f.mean()
    return f / np.max(np.abs(f))


def make_model(nx: int, nz_f: int, nz_s: int, *, h: float = 5.0, npd: int = 20,
               fpeak: float = 15.0, dt: float = 5e-4, nt: int = 2000, snapshot: Optional[int] = None,
               src_x: Optional[List[int]] = None, src_z: Optional[List[int]] = None,
               vp_f: float = 1500.0, rho_f: float = 1000.0,
               vp: float = 3000.0, vs: float = 1732.0, rho: float = 2000.0,
               amp: float = 0.0, wavelength: float = 600.0,
               perturb: float = 0.0, corr_len: float = 50.0, seed: int = 0,
               ppw: float = 8.0, npow: int = 2, rc: float = 1e-3, boundary_type: int = 2,
               flat_sides: bool = True,
               seafloor: Optional[Tuple[np.ndarray, np.ndarray]] = None) -> Model:
    """Builds a fluid-over-solid model: ``amp > 0`` gives a sinusoidal seafloor,
    ``seafloor = (g, dg)`` any other profile (perturbation per column and its
    derivative along xi). ``flat_sides`` holds the outer npd + 3 columns flat."""
    pad = npd + 3 if flat_sides else 0
    g, dg = seafloor if seafloor is not None else sinusoid_profile(nx, h, amp, wavelength, pad)
    g, dg = _flat_pads(np.asarray(g, np.float64), np.asarray(dg, np.float64), pad)
    top = npd + 3 if boundary_type == 1 else 3
    metric = _grid_metric(nx, nz_f, nz_s, npd, h, g, dg, top)
    solid_shape = (nz_s, nx)
    vp_s = np.full(solid_shape, vp)
    vs_s = np.full(solid_shape, vs)
    rho_s = np.full(solid_shape, rho)
    if perturb:
        rng = np.random.default_rng(seed)
        corr = corr_len / h
        vp_s *= 1.0 + perturb * _correlated_field(rng, solid_shape, corr)
        vs_s *= 1.0 + perturb * _correlated_field(rng, solid_shape, corr)
        rho_s *= 1.0 + perturb * _correlated_field(rng, solid_shape, corr)
    mu = rho_s * vs_s ** 2
    lam = rho_s * (vp_s ** 2 - 2.0 * vs_s ** 2)
    solid = {"C11": lam + 2.0 * mu, "C13": lam, "C33": lam + 2.0 * mu, "C55": mu, "rho": rho_s}
    fluid = {"K": np.full((nz_f, nx), rho_f * vp_f ** 2), "rho": np.full((nz_f, nx), rho_f)}
    vpmax = float(max(np.max(vp_s), vp_f))
    beta0 = round(min(float(np.min(vs_s)), vp_f) / (0.5 * ppw * h * fpeak), 4)
    if src_x is None:
        src_x = [nx // 2]
    if src_z is None:
        src_z = [max(3 + 3, nz_f - 1 - int(round(50.0 / h)))]
    return Model(nx=nx, nz_f=nz_f, nz_s=nz_s, h=h, fpeak=fpeak, dt=dt, nt=nt,
                 snapshot=snapshot if snapshot is not None else nt + 1,
                 src_x=list(src_x), src_z=list(src_z), npd=npd, npow=npow,
                 thickness=(npd - 1) * h, vp_max=vpmax, rc=rc, beta0=beta0,
                 fluid=fluid, solid=solid, metric=metric, boundary_type=boundary_type, pad=pad)


def _solid_metric(nx: int, nz: int, npd: int, h: float, amp: float,
                  wavelength: float, boundary_type: int = 2) -> Dict[str, np.ndarray]:
    """FP64 metric of z(xi, zeta) = h (zeta - 3) + amp sin(2 pi x / wavelength) w(zeta).

    boundary_type 2: a free surface with topography on row 3, w = cos^2 falling
    1 -> 0 between row 3 and b = nz - 4 - npd (flat below, so the bottom band is
    flat; ``model_SOLID_PANDF_wavy_if.py:113-121``). boundary_type 1 (CFS-PML on
    all four sides, no free surface): an undulation inside the grid,
    w = sin^2(pi t) between a = npd + 3 and b, zero in both PML bands so they
    are flat (``model_SOLID_PANDF_wavy_if.py:104-110``)."""
    zeta = np.arange(nz, dtype=np.float64)
    b = float(nz - 4 - npd)
    if boundary_type == 1:
        a = float(npd + 3)
        t = np.clip((zeta - a) / (b - a), 0.0, 1.0)
        inside = (t > 0.0) & (t < 1.0)
        w = np.sin(math.pi * t) ** 2
        dw = np.where(inside, math.pi / (b - a) * np.sin(2.0 * math.pi * t), 0.0)
    else:
        t = np.clip((zeta - 3.0) / (b - 3.0), 0.0, 1.0)
        w = np.cos(0.5 * math.pi * t) ** 2
        dw = np.where((t > 0.0) & (t < 1.0), -0.5 * math.pi / (b - 3.0) * np.sin(math.pi * t), 0.0)
    x = h * np.arange(nx, dtype=np.float64)
    s = np.sin(2.0 * math.pi * x / wavelength) if amp else np.zeros(nx)
    c = np.cos(2.0 * math.pi * x / wavelength) if amp else np.zeros(nx)
    z_xi = amp * (2.0 * math.pi * h / wavelength) * c[None, :] * w[:, None]
    z_ze = h + amp * s[None, :] * dw[:, None]
    if np.any(z_ze <= 0.0):
        raise ValueError("grid folds: z_zeta <= 0")
    J = h * z_ze
    return {"J": J, "xi_x": np.full((nz, nx), 1.0 / h), "xi_z": np.zeros((nz, nx)),
            "ze_x": -z_xi / J, "ze_z": h / J}


def make_solid_model(nx: int, nz: int, *, h: float = 5.0, npd: int = 20, fpeak: float = 15.0,
                     dt: float = 5e-4, nt: int = 2000, snapshot: Optional[int] = None,
                     src_x: Optional[List[int]] = None, src_z: Optional[List[int]] = None,
                     vp: float = 3000.0, vs: float = 1732.0, rho: float = 2000.0,
                     amp: float = 0.0, wavelength: float = 600.0, perturb: float = 0.0,
                     corr_len: float = 50.0, seed: int = 0, ppw: float = 8.0, npow: int = 2,
                     rc: float = 1e-3, boundary_type: int = 2) -> SolidModel:
    """A solid half-space with a free surface (flat, or with topography when amp > 0);
    with boundary_type 1 a solid with CFS-PML on all four sides (an undulating
    grid inside when amp > 0)."""
    metric = _solid_metric(nx, nz, npd, h, amp, wavelength, boundary_type)
    shape = (nz, nx)
    vp_s, vs_s, rho_s = np.full(shape, vp), np.full(shape, vs), np.full(shape, rho)
    if perturb:
        rng = np.random.default_rng(seed)
        corr = corr_len / h
        vp_s *= 1.0 + perturb * _correlated_field(rng, shape, corr)
        vs_s *= 1.0 + perturb * _correlated_field(rng, shape, corr)
        rho_s *= 1.0 + perturb * _correlated_field(rng, shape, corr)
    mu = rho_s * vs_s ** 2
    lam = rho_s * (vp_s ** 2 - 2.0 * vs_s ** 2)
    solid = {"C11": lam + 2.0 * mu, "C13": lam, "C33": lam + 2.0 * mu, "C55": mu, "rho": rho_s}
    beta0 = round(float(np.min(vs_s)) / (0.5 * ppw * h * fpeak), 4)
    return SolidModel(nx=nx, nz=nz, h=h, fpeak=fpeak, dt=dt, nt=nt,
                      snapshot=snapshot if snapshot is not None else nt + 1,
                      src_x=list(src_x if src_x is not None else [nx // 2]),
                      src_z=list(src_z if src_z is not None else [10]),
                      npd=npd, npow=npow, thickness=(npd - 1) * h,
                      vp_max=float(np.max(vp_s)), rc=rc, beta0=max(1.0, beta0),
                      solid=solid, metric=metric, boundary_type=boundary_type)


def beta0_rule(model: Model, fpeak: float, ppw: float = 8.0) -> float:
    """CFS-PML beta0 of the generators for a given Ricker frequency:
    min(vs, vp_fluid) / (0.5 ppw h fpeak) (``model_FANDS_PANDF_wavy.py:174-177``),
    never below 1."""
    vs_min = float(np.sqrt(np.min(model.solid["C55"] / model.solid["rho"])))
    vp_f = float(np.sqrt(np.min(model.fluid["K"] / model.fluid["rho"])))
    return max(1.0, round(min(vs_min, vp_f) / (0.5 * ppw * model.h * fpeak), 4))


# --- named workloads ---------------------------------------------------------

def flat_400x400(nt: int = 2000) -> Model:
    """400x400, h = 5 m, flat seafloor 1000 m below the free surface (global row 203),
    water 1500/1000 over vp 3000, vs 1732, rho 2000; 20-cell CFS-PML; 15 Hz Ricker
    50 m above the seafloor (column 200, fluid row 193); dt = 0.5 ms."""
    return make_model(400, 204, 197, h=5.0, npd=20, fpeak=15.0, dt=5e-4, nt=nt,
                      src_x=[200], src_z=[193])


def curvilinear(nx: int, nz: int, *, zeta0: Optional[int] = None, nt: int = 6000,
                dt: float = 4e-4, seed: int = 1, perturb: float = 0.05) -> Model:
    """Curvilinear forward model: sinusoidal seafloor 40 sin(2 pi x / 600 m) on global
    row ``zeta0`` (default: 1500 m below the free surface, row 303), blended into the
    grid, +-5% Gaussian-correlated vp/vs/rho (50 m), dt = 0.4 ms."""
    h = 5.0
    if zeta0 is None:
        zeta0 = min(303, nz // 2)
    nz_f = zeta0 + 1
    nz_s = nz - nz_f + 1
    return make_model(nx, nz_f, nz_s, h=h, npd=20, fpeak=15.0, dt=dt, nt=nt,
                      src_x=[nx // 2], src_z=[zeta0 - 10], amp=40.0, wavelength=600.0,
                      perturb=perturb, corr_len=50.0, seed=seed)


def layered(nx: int, nz: int, *, seed: int, nt: int = 2000, dt: float = 3e-4,
            vp_range=(1500.0, 4500.0), max_layers: int = 6) -> Model:
    """Water over a seeded stack of flat-lying solid layers (2..max_layers), vp
    rising with depth inside ``vp_range``, vs = vp / sqrt(3), Gardner density
    rho = 310 vp^0.25 (kg/m^3, vp in m/s), on a gently undulating seafloor
    (0..30 m amplitude) between 30% and 60% of the depth. dt = 0.3 ms keeps
    vp dt / h <= 0.27 at vp = 4500 m/s and h = 5 m."""
    rng = np.random.default_rng(seed)
    zeta0 = int(rng.integers(int(0.3 * nz), int(0.6 * nz) + 1))
    nz_f = zeta0 + 1
    nz_s = nz - nz_f + 1
    amp = float(rng.uniform(0.0, 30.0))
    m = make_model(nx, nz_f, nz_s, h=5.0, npd=20, fpeak=15.0, dt=dt, nt=nt,
                   src_x=[int(rng.integers(nx // 4, 3 * nx // 4))], src_z=[zeta0 - 10],
                   amp=amp, wavelength=600.0)
    nl = int(rng.integers(2, max_layers + 1))
    tops = np.sort(rng.choice(np.arange(1, nz_s - 1), size=nl - 1, replace=False))
    vps = np.sort(rng.uniform(max(vp_range[0], 1800.0), vp_range[1], size=nl))
    vp = np.empty((nz_s, nx))
    for k, v in enumerate(vps):
        lo = 0 if k == 0 else tops[k - 1]
        hi = nz_s if k == nl - 1 else tops[k]
        vp[lo:hi] = v
    vs = vp / math.sqrt(3.0)
    rho = 310.0 * vp ** 0.25
    mu = rho * vs ** 2
    lam = rho * (vp ** 2 - 2.0 * vs ** 2)
    m.solid = {"C11": lam + 2.0 * mu, "C13": lam, "C33": lam + 2.0 * mu, "C55": mu, "rho": rho}
    m.vp_max = float(max(vps.max(), vp_range[0]))
    m.beta0 = beta0_rule(m, m.fpeak)
    return m


def uneven_models(n: int = 32, seed: int = 3, nt: int = 2000) -> List[Model]:
    """``n`` layered models of seeded uneven sizes, nx in [400, 2000] and nz in
    [300, 1000] (multiples of 8)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nx = int(rng.integers(50, 251)) * 8
        nz = int(rng.integers(38, 126)) * 8
        out.append(layered(nx, nz, seed=seed * 1000 + k, nt=nt))
    return out


def curvilinear_1200x800(nt: int = 6000) -> Model:
    return curvilinear(1200, 800, nt=nt)


def curvilinear_4096x2048(nt: int = 6000) -> Model:
    """4096x2048 with the seafloor on the middle row (half fluid, half solid)."""
    return curvilinear(4096, 2048, zeta0=1023, nt=nt)


def _solid_velocities(m: Model) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    rho = m.solid["rho"]
    return np.sqrt(m.solid["C11"] / rho), np.sqrt(m.solid["C55"] / rho), rho


def _set_solid(m: Model, vp: np.ndarray, vs: np.ndarray, rho: np.ndarray) -> None:
    mu = rho * vs ** 2
    lam = rho * (vp ** 2 - 2.0 * vs ** 2)
    m.solid = {"C11": lam + 2.0 * mu, "C13": lam, "C33": lam + 2.0 * mu, "C55": mu, "rho": rho}


def adjoint_pair(nx: int = 800, nz: int = 400, *, nt: int = 4000, anomaly: float = 0.10,
                 radius: float = 60.0, depth: float = 150.0, smooth: float = 100.0,
                 seed: int = 1) -> Tuple[Model, Model]:
    """The true and initial models of the 800 x 400 adjoint-gradient workload.

    Both share the curvilinear grid and background of ``curvilinear`` (sinusoidal
    seafloor, +-5 % correlated perturbations, dt = 0.4 ms). The true model adds
    a Gaussian vs anomaly ``1 + anomaly * exp(-d^2 / radius^2)``, d the physical
    distance to a point ``depth`` metres below the seafloor under the middle
    column (vp and rho unchanged). The initial model is the true model's solid
    vp, vs and rho smoothed by a Gaussian of ``smooth`` metres (sigma), which
    removes the anomaly and most of the perturbations; the fluid is unchanged."""
    from scipy.ndimage import gaussian_filter

    true = curvilinear(nx, nz, nt=nt, seed=seed)
    vp, vs, rho = _solid_velocities(true)
    z0 = true.nz_f - 1
    xs = true.metric["x"][z0:]
    zs = true.metric["z"][z0:]
    xc = xs[0, nx // 2]
    zc = zs[0, nx // 2] + depth
    d2 = (xs - xc) ** 2 + (zs - zc) ** 2
    _set_solid(true, vp, vs * (1.0 + anomaly * np.exp(-d2 / radius ** 2)), rho)
    init = curvilinear(nx, nz, nt=nt, seed=seed)
    vp_t, vs_t, rho_t = _solid_velocities(true)
    sig = smooth / true.h
    _set_solid(init, *(gaussian_filter(a, sig, mode="nearest") for a in (vp_t, vs_t, rho_t)))
    for m in (true, init):
        m.vp_max = float(max(np.max(_solid_velocities(m)[0]), 1500.0))
        m.beta0 = beta0_rule(m, m.fpeak)
    init.vp_max = true.vp_max = max(true.vp_max, init.vp_max)
    init.beta0 = true.beta0 = min(true.beta0, init.beta0)
    return true, init


def rough_seafloor(nx: int = 8192, nz: int = 4096, *, nt: int = 8000, fpeak: float = 10.0,
                   hurst: float = 0.7, rms: float = 20.0, corr: float = 200.0, seed: int = 5,
                   nshots: int = 16, dt: float = 4e-4) -> Model:
    """The large batched-adjoint workload: an ``nx x nz`` grid (h = 5 m) with a
    seeded von Kármán rough seafloor (Hurst 0.7, rms 20 m, correlation 200 m) on
    the middle row, water over the elastic background of the flat model
    (vp 3000, vs 1732, rho 2000), a 10 Hz Ricker, and ``nshots`` sources evenly
    spaced 50 m above the seafloor. Flat side pads as every fluid-solid model."""
    npd = 20
    zeta0 = nz // 2 - 1
    nz_f = zeta0 + 1
    nz_s = nz - nz_f + 1
    pad = npd + 3
    g, dg = von_karman_profile(nx - 2 * pad, 5.0, hurst=hurst, rms=rms, corr=corr, seed=seed)
    gp = np.concatenate([np.full(pad, g[0]), g, np.full(pad, g[-1])])
    dgp = np.concatenate([np.zeros(pad), dg, np.zeros(pad)])
    xs = [int(round(pad + (k + 0.5) * (nx - 2 * pad) / nshots)) for k in range(nshots)]
    return make_model(nx, nz_f, nz_s, h=5.0, npd=npd, fpeak=fpeak, dt=dt, nt=nt,
                      src_x=xs, src_z=[zeta0 - 10] * nshots, seafloor=(gp, dgp))
