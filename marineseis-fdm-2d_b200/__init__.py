"""B200-native MarineSeis-FDM-2D time stepping: Python binding of libmfdm.so.

The compute path is the CUDA library built from ``csrc/`` for sm_100a
(``builder.build()``); this module only marshals arguments through ctypes. There
is no CPU fallback: if the library is missing or no GPU is present the calls
raise ``MfdmError``.

Mirrors the reference's interfaces for the fluid-solid PANDF path:

* ``Solver.from_json(path)``      MemManager(json) + grid_cp_h2d (src/elements.cu:64-183, 307-333)
* ``Solver.update_rk4(it)``       PmlFs::FluidSolid::update_RK4 (src/pml_fs_kernels.cu:765-868)
* ``Solver.step(n)``              the time loop of src/main.cu:136-213 (graph-captured)
* ``Solver.records()``            record/{solid_vx,solid_vz,fluid_p}.bin rows (src/main.cu:245-295)
* ``Solver.field(name)``          MemManager::U_cp_d2h (src/elements.cu:335-343)
* ``run_cli(json, out_root)``     ``main_debug <model.json> <out_root>`` (src/main.cu:58-216)
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmfdm.so")
CLI_PATH = os.path.join(HERE, "bin", "main_debug")

FIELDS = {"fluid_vx": 0, "fluid_vz": 1, "fluid_p": 2, "solid_vx": 3, "solid_vz": 4,
          "solid_sx": 5, "solid_sz": 6, "solid_sxz": 7}

# Entry points declared in include/mfdm.h (checked by the CPU test suite).
EXPORTS = ("mfdm_last_error", "mfdm_open_json", "mfdm_open_desc", "mfdm_load_desc", "mfdm_close",
           "mfdm_get_info", "mfdm_set_shot", "mfdm_update_rk4", "mfdm_step", "mfdm_time_steps",
           "mfdm_synchronize", "mfdm_get_records", "mfdm_get_field", "mfdm_set_field",
           "mfdm_run_cli", "mfdm_run_cli_batch", "mfdm_step_noalloc", "mfdm_open_batch", "mfdm_batch_reset",
           "mfdm_batch_get_records", "mfdm_batch_get_field", "mfdm_set_tile", "mfdm_autotune",
           "mfdm_group_open", "mfdm_group_step", "mfdm_group_time_steps", "mfdm_group_close",
           "mfdm_adjoint_forward", "mfdm_adjoint_backward", "mfdm_adjoint_set_memory",
           "mfdm_solid_open_json", "mfdm_solid_open_desc", "mfdm_solid_set_shot", "mfdm_solid_step",
           "mfdm_solid_time_steps", "mfdm_solid_get_records", "mfdm_solid_get_field",
           "mfdm_solid_get_info", "mfdm_solid_close", "mfdm_set_blocks_per_sm",
           "mfdm_adjoint_set_inner", "mfdm_adjoint_accumulate_grad_f32",
           "mfdm_dispersion_velocities", "mfdm_dispersion_image")

# Coefficient arrays the adjoint differentiates (mfdm_coef_grad order).
GRAD_COEFS = ("K", "rcp_rho_f", "C11", "C13", "C33", "C55", "rcp_rho_s")


class MfdmError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"mfdm error {code}: {message}")
        self.code = code


_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int)


class Desc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("nz_f", ctypes.c_int), ("nz_s", ctypes.c_int),
                ("fpeak", ctypes.c_float), ("dt", ctypes.c_float),
                ("nt", ctypes.c_int), ("snapshot", ctypes.c_int),
                ("npd", ctypes.c_int), ("npow", ctypes.c_int),
                ("thickness", ctypes.c_float), ("vp_max", ctypes.c_float),
                ("rc", ctypes.c_float), ("beta0", ctypes.c_float),
                ("nsrc", ctypes.c_int), ("src_x", _ip), ("src_z", _ip),
                ("K", _fp), ("rho_f", _fp), ("C11", _fp), ("C13", _fp), ("C33", _fp),
                ("C55", _fp), ("rho_s", _fp), ("J", _fp), ("xi_x", _fp), ("xi_z", _fp),
                ("ze_x", _fp), ("ze_z", _fp), ("boundary_type", ctypes.c_int)]


class Info(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("nz_f", ctypes.c_int), ("nz_s", ctypes.c_int),
                ("pitch", ctypes.c_int), ("nt", ctypes.c_int), ("snapshot", ctypes.c_int),
                ("gap", ctypes.c_int), ("nsrc", ctypes.c_int), ("shot", ctypes.c_int),
                ("step", ctypes.c_int), ("nsamples", ctypes.c_int),
                ("cells", ctypes.c_longlong), ("device_bytes", ctypes.c_longlong),
                ("nshots", ctypes.c_int), ("seg_rows", ctypes.c_int),
                ("blocks_per_sm", ctypes.c_int)]


class SolidDesc(ctypes.Structure):
    """mfdm_solid_desc: a solid-only model (calc_type 0) in caller memory."""
    _fields_ = [("nx", ctypes.c_int), ("nz", ctypes.c_int),
                ("fpeak", ctypes.c_float), ("dt", ctypes.c_float),
                ("nt", ctypes.c_int), ("snapshot", ctypes.c_int),
                ("npd", ctypes.c_int), ("npow", ctypes.c_int),
                ("thickness", ctypes.c_float), ("vp_max", ctypes.c_float),
                ("rc", ctypes.c_float), ("beta0", ctypes.c_float),
                ("nsrc", ctypes.c_int), ("src_x", _ip), ("src_z", _ip),
                ("C11", _fp), ("C13", _fp), ("C33", _fp), ("C55", _fp), ("rho", _fp),
                ("J", _fp), ("xi_x", _fp), ("xi_z", _fp), ("ze_x", _fp), ("ze_z", _fp),
                ("boundary_type", ctypes.c_int)]


class CoefGrad(ctypes.Structure):
    """mfdm_coef_grad: host [rows][nx] float64 arrays (NULL: not wanted)."""
    _fields_ = [(k, ctypes.POINTER(ctypes.c_double)) for k in GRAD_COEFS]


class Shot(ctypes.Structure):
    """mfdm_shot: one shot of a batch (source cell, Ricker peak frequency, PML beta0)."""
    _fields_ = [("src_x", ctypes.c_int), ("src_z", ctypes.c_int), ("fpeak", ctypes.c_float),
                ("beta0", ctypes.c_float)]


class DeviceModel(ctypes.Structure):
    """mfdm_device_model: device pointers for mfdm_step_noalloc (no allocation)."""
    _fields_ = [("nx", ctypes.c_int), ("nz_f", ctypes.c_int), ("nz_s", ctypes.c_int),
                ("fpeak", ctypes.c_float), ("dt", ctypes.c_float),
                ("npd", ctypes.c_int), ("npow", ctypes.c_int),
                ("thickness", ctypes.c_float), ("vp_max", ctypes.c_float),
                ("rc", ctypes.c_float), ("beta0", ctypes.c_float),
                ("src_x", ctypes.c_int), ("src_z", ctypes.c_int)] + [
        (n, ctypes.c_void_p) for n in ("K", "rho_f", "C11", "C13", "C33", "C55", "rho_s", "J",
                                       "xi_x", "xi_z", "ze_x", "ze_z", "vx_f", "vz_f", "p_f",
                                       "vx_s", "vz_s", "sx_s", "sz_s", "sxz_s")]


_lib = None


def load_library(path: str = LIB_PATH):
    """Loads libmfdm.so (raises if it was not built; there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise MfdmError(-1, f"{path} is missing: build it with marineseis-fdm-2d_b200/builder.py")
    lib = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    sig = {
        "mfdm_last_error": (ctypes.c_char_p, []),
        "mfdm_open_json": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(vp)]),
        "mfdm_open_desc": (ctypes.c_int, [ctypes.POINTER(Desc), ctypes.c_int, ctypes.POINTER(vp)]),
        "mfdm_load_desc": (ctypes.c_int, [vp, ctypes.POINTER(Desc)]),
        "mfdm_close": (ctypes.c_int, [vp]),
        "mfdm_get_info": (ctypes.c_int, [vp, ctypes.POINTER(Info)]),
        "mfdm_set_shot": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
        "mfdm_update_rk4": (ctypes.c_int, [vp, ctypes.c_int, vp]),
        "mfdm_step": (ctypes.c_int, [vp, ctypes.c_int]),
        "mfdm_time_steps": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, _fp, _fp]),
        "mfdm_synchronize": (ctypes.c_int, [vp]),
        "mfdm_get_records": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, _fp, _fp, _fp]),
        "mfdm_get_field": (ctypes.c_int, [vp, ctypes.c_int, _fp]),
        "mfdm_set_field": (ctypes.c_int, [vp, ctypes.c_int, _fp]),
        "mfdm_run_cli": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]),
        "mfdm_run_cli_batch": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]),
        "mfdm_step_noalloc": (ctypes.c_int, [ctypes.POINTER(DeviceModel), ctypes.c_int,
                                             ctypes.c_int, vp]),
        "mfdm_open_batch": (ctypes.c_int, [ctypes.POINTER(Desc), ctypes.c_int,
                                           ctypes.POINTER(Shot), ctypes.c_int, ctypes.POINTER(vp)]),
        "mfdm_batch_reset": (ctypes.c_int, [vp]),
        "mfdm_batch_get_records": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                  _fp, _fp, _fp]),
        "mfdm_batch_get_field": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, _fp]),
        "mfdm_set_tile": (ctypes.c_int, [vp, ctypes.c_int]),
        "mfdm_set_blocks_per_sm": (ctypes.c_int, [vp, ctypes.c_int]),
        "mfdm_autotune": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int)]),
        "mfdm_group_open": (ctypes.c_int, [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(vp)]),
        "mfdm_group_step": (ctypes.c_int, [vp, ctypes.c_int]),
        "mfdm_group_time_steps": (ctypes.c_int, [vp, ctypes.c_int, _fp]),
        "mfdm_group_close": (ctypes.c_int, [vp]),
        "mfdm_adjoint_forward": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
        "mfdm_adjoint_set_memory": (ctypes.c_int, [vp, ctypes.c_longlong]),
        "mfdm_adjoint_set_inner": (ctypes.c_int, [vp, ctypes.c_int]),
        "mfdm_solid_open_json": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(vp)]),
        "mfdm_solid_open_desc": (ctypes.c_int, [ctypes.POINTER(SolidDesc), ctypes.c_int,
                                                ctypes.POINTER(vp)]),
        "mfdm_solid_set_shot": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
        "mfdm_solid_step": (ctypes.c_int, [vp, ctypes.c_int]),
        "mfdm_solid_time_steps": (ctypes.c_int, [vp, ctypes.c_int, _fp]),
        "mfdm_solid_get_records": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, _fp]),
        "mfdm_solid_get_field": (ctypes.c_int, [vp, ctypes.c_int, _fp]),
        "mfdm_solid_get_info": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_int)]),
        "mfdm_solid_close": (ctypes.c_int, [vp]),
        "mfdm_adjoint_backward": (ctypes.c_int, [vp, _fp, _fp, _fp, ctypes.POINTER(CoefGrad)]),
        "mfdm_adjoint_accumulate_grad_f32": (ctypes.c_int, [vp, vp, vp]),
        "mfdm_dispersion_velocities": (ctypes.c_int, [ctypes.c_double] * 3),
        "mfdm_dispersion_image": (ctypes.c_int, [_fp, ctypes.c_int, ctypes.c_int,
                                                 ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                                                 ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                 _fp, ctypes.c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(rc: int):
    if rc != 0:
        msg = load_library().mfdm_last_error().decode(errors="replace")
        raise MfdmError(rc, msg)


def _f32(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def make_desc(model):
    """mfdm_desc for a modelgen.Model; returns (desc, arrays kept alive)."""
    keep = []

    def ptr(a):
        a = _f32(a)
        keep.append(a)
        return a.ctypes.data_as(_fp)

    d = Desc()
    d.nx, d.nz_f, d.nz_s = model.nx, model.nz_f, model.nz_s
    d.fpeak, d.dt, d.nt, d.snapshot = model.fpeak, model.dt, model.nt, model.snapshot
    d.npd, d.npow, d.thickness = model.npd, model.npow, model.thickness
    d.vp_max, d.rc, d.beta0 = model.vp_max, model.rc, model.beta0
    sx = np.ascontiguousarray(model.src_x, dtype=np.int32)
    sz = np.ascontiguousarray(model.src_z, dtype=np.int32)
    keep += [sx, sz]
    d.nsrc, d.src_x, d.src_z = len(sx), sx.ctypes.data_as(_ip), sz.ctypes.data_as(_ip)
    d.K, d.rho_f = ptr(model.fluid["K"]), ptr(model.fluid["rho"])
    d.C11, d.C13 = ptr(model.solid["C11"]), ptr(model.solid["C13"])
    d.C33, d.C55, d.rho_s = ptr(model.solid["C33"]), ptr(model.solid["C55"]), ptr(model.solid["rho"])
    d.J, d.xi_x, d.xi_z = ptr(model.metric["J"]), ptr(model.metric["xi_x"]), ptr(model.metric["xi_z"])
    d.ze_x, d.ze_z = ptr(model.metric["ze_x"]), ptr(model.metric["ze_z"])
    d.boundary_type = int(getattr(model, "boundary_type", 2))
    return d, keep


class Solver:
    """One model resident on one GPU (an opaque libmfdm handle)."""

    def __init__(self, handle: ctypes.c_void_p):
        self._h = handle
        self._lib = load_library()
        self.info()

    # -- construction -------------------------------------------------------
    @classmethod
    def from_json(cls, path: str, device: int = 0) -> "Solver":
        h = ctypes.c_void_p()
        _check(load_library().mfdm_open_json(os.fsencode(path), device, ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_model(cls, model, device: int = 0) -> "Solver":
        """From a modelgen.Model held in host memory (no files)."""
        d, keep = make_desc(model)
        h = ctypes.c_void_p()
        _check(load_library().mfdm_open_desc(ctypes.byref(d), device, ctypes.byref(h)))
        del keep
        return cls(h)

    def load_model(self, model):
        """Uploads a model of the same shape into this handle (mfdm_load_desc)."""
        d, keep = make_desc(model)
        _check(self._lib.mfdm_load_desc(self._h, ctypes.byref(d)))
        del keep

    def close(self):
        if self._h:
            self._lib.mfdm_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- queries ------------------------------------------------------------
    def info(self) -> Dict[str, int]:
        i = Info()
        _check(self._lib.mfdm_get_info(self._h, ctypes.byref(i)))
        return {k: getattr(i, k) for k, _ in Info._fields_}

    # -- time stepping ------------------------------------------------------
    def set_shot(self, isrc: int = 0, reset: bool = True):
        _check(self._lib.mfdm_set_shot(self._h, int(isrc), 1 if reset else 0))

    def update_rk4(self, it: int, stream: Optional[int] = None):
        """One RK4 step for time index ``it`` (asynchronous on ``stream`` or the handle's)."""
        _check(self._lib.mfdm_update_rk4(self._h, int(it), ctypes.c_void_p(stream or 0)))

    def step(self, nsteps: int):
        _check(self._lib.mfdm_step(self._h, int(nsteps)))

    def time_steps(self, nsteps: int, per_kernel: bool = False):
        """Runs nsteps and returns (total_ms, per-kernel ms [4 stages + filter] or None),
        measured with CUDA events on the handle's stream."""
        total = ctypes.c_float()
        k = (ctypes.c_float * 5)()
        _check(self._lib.mfdm_time_steps(self._h, int(nsteps), 1 if per_kernel else 0,
                                         ctypes.byref(total), k))
        return total.value, (list(k) if per_kernel else None)

    def synchronize(self):
        _check(self._lib.mfdm_synchronize(self._h))

    # -- adjoint ----------------------------------------------------------------
    def adjoint_memory(self, nbytes: int):
        """Device memory the adjoint may use to keep whole checkpoint segments'
        stage inputs from the forward pass (mfdm_adjoint_set_memory; 0: recompute all)."""
        _check(self._lib.mfdm_adjoint_set_memory(self._h, int(nbytes)))

    def adjoint_inner(self, inner_every: int):
        """Second checkpoint level of the backward pass (mfdm_adjoint_set_inner; 0: one level)."""
        _check(self._lib.mfdm_adjoint_set_inner(self._h, int(inner_every)))

    def adjoint_forward(self, nsteps: int, ckpt_every: int = 50) -> Dict[str, np.ndarray]:
        """Runs the current shot from rest with checkpoints (mfdm_adjoint_forward)
        and returns its records {'svx', 'svz', 'fp'}: [samples][nx]."""
        _check(self._lib.mfdm_adjoint_forward(self._h, int(nsteps), int(ckpt_every)))
        return self.records()

    def adjoint_backward(self, residual: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
        """Gradients of sum(residual . records) with respect to the coefficient
        arrays (mfdm_adjoint_backward): {'K', 'rcp_rho_f'}: [nz_f][nx] and
        {'C11', 'C13', 'C33', 'C55', 'rcp_rho_s'}: [nz_s][nx], float64."""
        info = self.info()
        out = {k: np.zeros((info["nz_f"] if k in ("K", "rcp_rho_f") else info["nz_s"], info["nx"]))
               for k in GRAD_COEFS}
        g = CoefGrad(*[out[k].ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for k in GRAD_COEFS])
        self._backward(residual, ctypes.byref(g))
        return out

    def adjoint_backward_only(self, residual: Dict[str, np.ndarray]):
        """mfdm_adjoint_backward without copying the gradient to the host: it
        stays on the device for adjoint_accumulate_grad."""
        self._backward(residual, None)

    def _backward(self, residual, grad):
        nx = self.info()["nx"]
        keep = []

        def res(name):
            a = residual.get(name)
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float32)
            if a.ndim != 2 or a.shape[1] != nx:
                raise ValueError(f"residual {name} must be [samples][{nx}]")
            keep.append(a)
            return a.ctypes.data_as(_fp)

        _check(self._lib.mfdm_adjoint_backward(self._h, res("svx"), res("svz"), res("fp"), grad))

    def adjoint_accumulate_grad(self, dst, stream: Optional[int] = None):
        """Adds the last backward pass's gradient, rounded to FP32, to the device
        buffer `dst` (a CUDA torch tensor of (2 nz_f + 5 nz_s) x nx float32, the
        seven GRAD_COEFS arrays packed) on `stream` (a CUDA stream handle; None:
        the legacy default stream), without a host round trip
        (mfdm_adjoint_accumulate_grad_f32)."""
        info = self.info()
        need = (2 * info["nz_f"] + 5 * info["nz_s"]) * info["nx"]
        if (not getattr(dst, "is_cuda", False) or dst.dtype.itemsize != 4 or dst.numel() != need
                or not dst.is_contiguous()):
            raise ValueError(f"dst must be a contiguous CUDA float32 tensor of {need} elements")
        _check(self._lib.mfdm_adjoint_accumulate_grad_f32(self._h, ctypes.c_void_p(dst.data_ptr()),
                                                          ctypes.c_void_p(stream or 0)))

    # -- tile shape -----------------------------------------------------------
    def set_tile(self, seg_rows: int):
        """Rows per segment block of the stage launches (multiple of 4 in [4, 128]; 0: 24)."""
        _check(self._lib.mfdm_set_tile(self._h, int(seg_rows)))

    def set_blocks_per_sm(self, blocks: int):
        """Stage kernel build: 2 or 3 resident blocks per SM (TMA rings), 4 (tiles), 0 the
        default 3 (mfdm_set_blocks_per_sm)."""
        _check(self._lib.mfdm_set_blocks_per_sm(self._h, int(blocks)))

    def autotune(self) -> int:
        """Times the candidate segment heights, keeps the fastest and returns it.
        Leaves every shot at rest at step 0 (mfdm_autotune)."""
        seg = ctypes.c_int()
        _check(self._lib.mfdm_autotune(self._h, ctypes.byref(seg)))
        return seg.value

    # -- data out -----------------------------------------------------------
    def records(self, first: int = 0, count: Optional[int] = None) -> Dict[str, np.ndarray]:
        info = self.info()
        if count is None:
            count = info["nsamples"] - first
        nx = info["nx"]
        out = {k: np.zeros((count, nx), dtype=np.float32) for k in ("svx", "svz", "fp")}
        _check(self._lib.mfdm_get_records(self._h, int(first), int(count),
                                          out["svx"].ctypes.data_as(_fp),
                                          out["svz"].ctypes.data_as(_fp),
                                          out["fp"].ctypes.data_as(_fp)))
        return out

    def field(self, name: str) -> np.ndarray:
        info = self.info()
        fid = FIELDS[name]
        rows = info["nz_f"] if fid < 3 else info["nz_s"]
        out = np.zeros((rows, info["nx"]), dtype=np.float32)
        _check(self._lib.mfdm_get_field(self._h, fid, out.ctypes.data_as(_fp)))
        return out

    def set_field(self, name: str, values: np.ndarray):
        a = _f32(values)
        _check(self._lib.mfdm_set_field(self._h, FIELDS[name], a.ctypes.data_as(_fp)))


class Batch(Solver):
    """Shots of one model stepped together (mfdm_open_batch): one launch per RK
    stage covers every shot. ``shots`` is a sequence of (src_x, src_z, fpeak,
    beta0); every shot starts from rest."""

    @classmethod
    def from_model(cls, model, shots, device: int = 0) -> "Batch":
        d, keep = make_desc(model)
        arr = (Shot * len(shots))(*[Shot(int(x), int(z), float(f), float(b))
                                    for x, z, f, b in shots])
        h = ctypes.c_void_p()
        _check(load_library().mfdm_open_batch(ctypes.byref(d), len(shots), arr, device,
                                              ctypes.byref(h)))
        del keep
        return cls(h)

    def reset(self):
        _check(self._lib.mfdm_batch_reset(self._h))

    def set_shot(self, isrc: int = 0, reset: bool = True):
        raise MfdmError(-1, "a batch runs its own shots: use reset()")

    def records(self, first: int = 0, count: Optional[int] = None,
                shot: int = 0) -> Dict[str, np.ndarray]:
        info = self.info()
        if count is None:
            count = info["nsamples"] - first
        nx = info["nx"]
        out = {k: np.zeros((count, nx), dtype=np.float32) for k in ("svx", "svz", "fp")}
        _check(self._lib.mfdm_batch_get_records(self._h, int(shot), int(first), int(count),
                                                out["svx"].ctypes.data_as(_fp),
                                                out["svz"].ctypes.data_as(_fp),
                                                out["fp"].ctypes.data_as(_fp)))
        return out

    def field(self, name: str, shot: int = 0) -> np.ndarray:
        info = self.info()
        fid = FIELDS[name]
        rows = info["nz_f"] if fid < 3 else info["nz_s"]
        out = np.zeros((rows, info["nx"]), dtype=np.float32)
        _check(self._lib.mfdm_batch_get_field(self._h, int(shot), fid, out.ctypes.data_as(_fp)))
        return out


class SolidSolver:
    """A solid-only model with a free surface (mfdm_solid_*; the reference's
    PmlFs::SolidOnly, calc_type 0)."""

    def __init__(self, handle: ctypes.c_void_p):
        self._lib = load_library()
        self._h = handle

    @classmethod
    def from_json(cls, path: str, device: int = 0) -> "SolidSolver":
        h = ctypes.c_void_p()
        _check(load_library().mfdm_solid_open_json(os.fsencode(path), device, ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_model(cls, model, device: int = 0) -> "SolidSolver":
        """From a modelgen.SolidModel (arrays read in place, float32)."""
        keep = []

        def ptr(a):
            a = _f32(a)
            keep.append(a)
            return a.ctypes.data_as(_fp)

        d = SolidDesc()
        d.nx, d.nz = model.nx, model.nz
        d.fpeak, d.dt, d.nt, d.snapshot = model.fpeak, model.dt, model.nt, model.snapshot
        d.npd, d.npow, d.thickness = model.npd, model.npow, model.thickness
        d.vp_max, d.rc, d.beta0 = model.vp_max, model.rc, model.beta0
        sx = np.ascontiguousarray(model.src_x, dtype=np.int32)
        sz = np.ascontiguousarray(model.src_z, dtype=np.int32)
        keep += [sx, sz]
        d.nsrc, d.src_x, d.src_z = len(sx), sx.ctypes.data_as(_ip), sz.ctypes.data_as(_ip)
        d.C11, d.C13 = ptr(model.solid["C11"]), ptr(model.solid["C13"])
        d.C33, d.C55, d.rho = ptr(model.solid["C33"]), ptr(model.solid["C55"]), ptr(model.solid["rho"])
        d.J, d.xi_x, d.xi_z = ptr(model.metric["J"]), ptr(model.metric["xi_x"]), ptr(model.metric["xi_z"])
        d.ze_x, d.ze_z = ptr(model.metric["ze_x"]), ptr(model.metric["ze_z"])
        d.boundary_type = int(getattr(model, "boundary_type", 2))
        h = ctypes.c_void_p()
        _check(load_library().mfdm_solid_open_desc(ctypes.byref(d), device, ctypes.byref(h)))
        return cls(h)

    def info(self) -> Dict[str, int]:
        v = [ctypes.c_int() for _ in range(4)]
        _check(self._lib.mfdm_solid_get_info(self._h, *[ctypes.byref(x) for x in v]))
        return dict(zip(("nx", "nz", "gap", "step"), [x.value for x in v]))

    def set_shot(self, isrc: int = 0, reset: bool = True):
        _check(self._lib.mfdm_solid_set_shot(self._h, int(isrc), 1 if reset else 0))

    def step(self, nsteps: int):
        _check(self._lib.mfdm_solid_step(self._h, int(nsteps)))

    def time_steps(self, nsteps: int) -> float:
        total = ctypes.c_float()
        _check(self._lib.mfdm_solid_time_steps(self._h, int(nsteps), ctypes.byref(total)))
        return total.value

    def records(self) -> Dict[str, np.ndarray]:
        """{'svz': solid vz on row 3, [samples][nx]}."""
        i = self.info()
        ns = -(-i["step"] // i["gap"])
        out = np.zeros((ns, i["nx"]), dtype=np.float32)
        _check(self._lib.mfdm_solid_get_records(self._h, 0, ns, out.ctypes.data_as(_fp)))
        return {"svz": out}

    def field(self, name: str) -> np.ndarray:
        i = self.info()
        out = np.zeros((i["nz"], i["nx"]), dtype=np.float32)
        _check(self._lib.mfdm_solid_get_field(self._h, FIELDS[name], out.ctypes.data_as(_fp)))
        return out

    def close(self):
        if self._h:
            self._lib.mfdm_solid_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Group:
    """Models of different sizes stepped together through one captured graph
    (mfdm_group_*). The solvers stay owned by the caller and must stay open."""

    def __init__(self, solvers):
        self._lib = load_library()
        self._solvers = list(solvers)
        arr = (ctypes.c_void_p * len(self._solvers))(*[s._h for s in self._solvers])
        h = ctypes.c_void_p()
        _check(self._lib.mfdm_group_open(arr, len(self._solvers), ctypes.byref(h)))
        self._h = h

    def step(self, nsteps: int):
        _check(self._lib.mfdm_group_step(self._h, int(nsteps)))

    def time_steps(self, nsteps: int) -> float:
        """Steps every model and returns the device time of the whole run (ms)."""
        total = ctypes.c_float()
        _check(self._lib.mfdm_group_time_steps(self._h, int(nsteps), ctypes.byref(total)))
        return total.value

    def close(self):
        if self._h:
            self._lib.mfdm_group_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def step_noalloc(dm: DeviceModel, it: int, nsteps: int, stream: Optional[int] = None):
    """mfdm_step_noalloc: steps device-resident arrays without any allocation."""
    _check(load_library().mfdm_step_noalloc(ctypes.byref(dm), int(it), int(nsteps),
                                            ctypes.c_void_p(stream or 0)))


def dispersion_image(gather: np.ndarray, offsets, fs: float, c_min: float, c_max: float,
                     dc: float, device: int = 0):
    """Phase-shift dispersion image of a gather [nt][ntr] on the GPU
    (mfdm_dispersion_image; the reference's tools/test.py:50-98). Returns
    (frequencies [nf], velocities [nv], amplitude [nf][nv])."""
    lib = load_library()
    g = np.ascontiguousarray(gather, dtype=np.float32)
    if g.ndim != 2:
        raise ValueError("gather must have shape (nt, number_of_receivers)")
    x = np.ascontiguousarray(offsets, dtype=np.float64)
    if x.ndim != 1 or x.size != g.shape[1]:
        raise ValueError("there must be exactly one offset for each trace")
    nv = lib.mfdm_dispersion_velocities(c_min, c_max, dc)
    if nv <= 0:
        raise MfdmError(-1, "velocities must satisfy 0 < c_min <= c_max and dc > 0")
    nt = g.shape[0]
    amp = np.zeros((nt // 2 + 1, nv), dtype=np.float32)
    _check(lib.mfdm_dispersion_image(g.ctypes.data_as(_fp), nt, g.shape[1],
                                     x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), fs, c_min,
                                     c_max, dc, amp.ctypes.data_as(_fp), int(device)))
    freqs = np.arange(nt // 2 + 1) * (fs / nt)
    vels = c_min + dc * np.arange(nv)
    return freqs, vels, amp


def run_cli(json_path: str, out_root: str, device: int = 0):
    """In-process equivalent of ``main_debug <model.json> <out_root>``."""
    _check(load_library().mfdm_run_cli(os.fsencode(json_path), os.fsencode(out_root), device))


def run_cli_batch(json_path: str, out_root: str, device: int = 0):
    """Every source of the JSON as one batch, each shot from rest (mfdm_run_cli_batch)."""
    _check(load_library().mfdm_run_cli_batch(os.fsencode(json_path), os.fsencode(out_root), device))


def build(verbose: bool = False, force: bool = False) -> str:
    """Compiles libmfdm.so and bin/main_debug for sm_100a (see builder.py)."""
    from . import builder
    return builder.build(verbose=verbose, force=force)
