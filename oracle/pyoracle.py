"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py, never by the product package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Dict, Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)


class _Model(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("nz_f", ctypes.c_int), ("nz_s", ctypes.c_int),
                ("npd", ctypes.c_int), ("npow", ctypes.c_int),
                ("fpeak", ctypes.c_double), ("dt", ctypes.c_double),
                ("thickness", ctypes.c_double), ("vp_max", ctypes.c_double),
                ("rc", ctypes.c_double), ("beta0", ctypes.c_double),
                ("src_x", ctypes.c_int), ("src_z", ctypes.c_int),
                ("K", _dp), ("rho_f", _dp),
                ("C11", _dp), ("C13", _dp), ("C33", _dp), ("C55", _dp), ("rho_s", _dp),
                ("J", _dp), ("xi_x", _dp), ("xi_z", _dp), ("ze_x", _dp), ("ze_z", _dp),
                ("cpml", ctypes.c_int)]


def build() -> str:
    """Compiles liboracle.so with the recipe in oracle/Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE, "oracle"], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = ctypes.CDLL(_LIB)
        _lib.orc_forward.restype = ctypes.c_int
        _lib.orc_forward.argtypes = [ctypes.POINTER(_Model), ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, _dp, _dp, _dp, _dp, _dp, ctypes.c_int]
        _lib.orc_forward_solid.restype = ctypes.c_int
        _lib.orc_forward_solid.argtypes = [ctypes.POINTER(_Model), ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, _dp, _dp, ctypes.c_int]
        _lib.orc_max_threads.restype = ctypes.c_int
        _lib.orc_create.restype = ctypes.c_void_p
        _lib.orc_create.argtypes = [ctypes.POINTER(_Model), ctypes.c_int]
        _lib.orc_step.restype = ctypes.c_int
        _lib.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        _lib.orc_destroy.restype = None
        _lib.orc_destroy.argtypes = [ctypes.c_void_p]
    return _lib


def _ptr(a: Optional[np.ndarray]):
    return a.ctypes.data_as(_dp) if a is not None else None


def forward(model, nsteps: int, gap: int, precision: int = 32, shot: int = 0,
            final_fields: bool = False, nthreads: int = 0,
            round_inputs: bool = True) -> Dict[str, np.ndarray]:
    """Runs the oracle from a zero wavefield for ``nsteps`` steps.

    ``model`` is a modelgen.Model. ``round_inputs`` rounds every array to
    float32 first (the inputs the reference reads from its .bin files);
    with False the FP64 oracle sees the FP64 metric of the generator.
    Returns records ``svx, svz, fp`` of shape [ceil(nsteps/gap)][nx] and,
    when asked, the final ``fluid`` [3][nz_f][nx] and ``solid`` [5][nz_s][nx].
    """
    m, keep = _model_struct(model, shot, round_inputs)
    ns = -(-nsteps // gap) if gap > 0 else 0
    out = {k: np.zeros((ns, model.nx)) for k in ("svx", "svz", "fp")}
    fl = np.zeros((3, model.nz_f, model.nx)) if final_fields else None
    so = np.zeros((5, model.nz_s, model.nx)) if final_fields else None
    rc = lib().orc_forward(ctypes.byref(m), int(precision), int(nsteps), int(gap),
                           _ptr(out["svx"]), _ptr(out["svz"]), _ptr(out["fp"]),
                           _ptr(fl), _ptr(so), int(nthreads))
    if rc != 0:
        raise RuntimeError(f"oracle failed ({rc})")
    if final_fields:
        out["fluid"], out["solid"] = fl, so
    return out


def _model_struct(model, shot=0, round_inputs=True):
    keep = []

    def arr(a):
        a = np.asarray(a, dtype=np.float64)
        if round_inputs:
            a = a.astype(np.float32).astype(np.float64)
        a = np.ascontiguousarray(a)
        keep.append(a)
        return _ptr(a)

    m = _Model()
    m.nx, m.nz_f, m.nz_s = model.nx, model.nz_f, model.nz_s
    m.npd, m.npow = model.npd, model.npow
    m.fpeak, m.dt, m.thickness = model.fpeak, model.dt, model.thickness
    m.vp_max, m.rc, m.beta0 = model.vp_max, model.rc, model.beta0
    m.src_x, m.src_z = model.src_x[shot], model.src_z[shot]
    m.K, m.rho_f = arr(model.fluid["K"]), arr(model.fluid["rho"])
    m.C11, m.C13 = arr(model.solid["C11"]), arr(model.solid["C13"])
    m.C33, m.C55 = arr(model.solid["C33"]), arr(model.solid["C55"])
    m.rho_s = arr(model.solid["rho"])
    m.J, m.xi_x, m.xi_z = arr(model.metric["J"]), arr(model.metric["xi_x"]), arr(model.metric["xi_z"])
    m.ze_x, m.ze_z = arr(model.metric["ze_x"]), arr(model.metric["ze_z"])
    m.cpml = 1 if getattr(model, "boundary_type", 2) == 1 else 0
    return m, keep


def forward_solid(model, nsteps: int, gap: int, precision: int = 32, shot: int = 0,
                  final_fields: bool = False, nthreads: int = 0,
                  round_inputs: bool = True) -> Dict[str, np.ndarray]:
    """Solid-only oracle for a modelgen.SolidModel, from rest: PmlFs::SolidOnly
    (boundary_type 2, free surface on top) or Cpml::SolidOnly (boundary_type 1,
    CFS-PML on all four sides).

    Returns the record ``svz`` (solid vz on row 3; row 30 with boundary_type 1)
    [ceil(nsteps/gap)][nx] and, when asked, the final ``solid`` [5][nz][nx]
    (vx, vz, sx, sz, sxz)."""
    keep = []

    def arr(a):
        a = np.asarray(a, dtype=np.float64)
        if round_inputs:
            a = a.astype(np.float32).astype(np.float64)
        a = np.ascontiguousarray(a)
        keep.append(a)
        return _ptr(a)

    m = _Model()
    m.nx, m.nz_f, m.nz_s = model.nx, 0, model.nz
    m.npd, m.npow = model.npd, model.npow
    m.fpeak, m.dt, m.thickness = model.fpeak, model.dt, model.thickness
    m.vp_max, m.rc, m.beta0 = model.vp_max, model.rc, model.beta0
    m.src_x, m.src_z = model.src_x[shot], model.src_z[shot]
    m.C11, m.C13 = arr(model.solid["C11"]), arr(model.solid["C13"])
    m.C33, m.C55 = arr(model.solid["C33"]), arr(model.solid["C55"])
    m.rho_s = arr(model.solid["rho"])
    m.J, m.xi_x, m.xi_z = arr(model.metric["J"]), arr(model.metric["xi_x"]), arr(model.metric["xi_z"])
    m.ze_x, m.ze_z = arr(model.metric["ze_x"]), arr(model.metric["ze_z"])
    m.cpml = 1 if getattr(model, "boundary_type", 2) == 1 else 0
    ns = -(-nsteps // gap) if gap > 0 else 0
    rec = np.zeros((ns, model.nx))
    so = np.zeros((5, model.nz, model.nx)) if final_fields else None
    rc = lib().orc_forward_solid(ctypes.byref(m), int(precision), int(nsteps), int(gap), _ptr(rec),
                                 _ptr(so), int(nthreads))
    if rc != 0:
        raise RuntimeError(f"oracle failed ({rc})")
    out = {"svz": rec}
    if final_fields:
        out["solid"] = so
    return out


class Stepper:
    """Persistent oracle state for timing the CPU restatement step by step."""

    def __init__(self, model, precision: int = 32, shot: int = 0):
        m, keep = _model_struct(model, shot, True)
        self._h = lib().orc_create(ctypes.byref(m), int(precision))
        if not self._h:
            raise RuntimeError("oracle create failed")

    def step(self, nsteps: int, nthreads: int = 0):
        if lib().orc_step(self._h, int(nsteps), int(nthreads)) != 0:
            raise RuntimeError("oracle step failed")

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def record_gap(dt: float) -> int:
    """Record interval of the reference CLI: (int)(1e-3 / float(dt) + 0.5) (src/main.cu:92)."""
    return int(1e-3 / float(np.float32(dt)) + 0.5)


def max_threads() -> int:
    return lib().orc_max_threads()
