"""Golden cases: seeded models whose records were produced by the reference's
own CUDA build (oracle/_ref/main_debug, compiled from the reference sources for
sm_100a) on a B200. make_golden.py writes the fixtures; the tests regenerate the
same models from these definitions and compare against the stored records.
"""
from __future__ import annotations

import importlib
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
modelgen = importlib.import_module("marineseis-fdm-2d_b200.modelgen")

GOLDEN_DIR = os.path.dirname(os.path.abspath(__file__))


def flat_small():
    """120 x 107 flat seafloor, 10-cell PML, 25 Hz, dt 0.5 ms, 600 steps."""
    return modelgen.make_model(120, 48, 60, npd=10, fpeak=25.0, dt=5e-4, nt=600,
                               src_x=[60], src_z=[40])


def curv_small():
    """128 x 115 sinusoidal seafloor + 5% perturbations, dt 0.4 ms (record gap 3), 500 steps."""
    return modelgen.make_model(128, 52, 64, npd=12, fpeak=25.0, dt=4e-4, nt=500,
                               src_x=[70], src_z=[44], amp=20.0, wavelength=300.0,
                               perturb=0.05, seed=3)


def shallow_src():
    """Source 2 rows below the free surface (source cells on the surface row), 300 steps."""
    return modelgen.make_model(96, 40, 48, npd=8, fpeak=30.0, dt=4e-4, nt=300,
                               src_x=[30], src_z=[5], amp=10.0, wavelength=200.0,
                               perturb=0.03, seed=7)


def flat_400x400():
    """The 400x400 flat-seafloor forward model, 2000 steps."""
    return modelgen.flat_400x400(nt=2000)


def curvilinear_1200x800():
    """The 1200x800 curvilinear forward model, 6000 steps."""
    return modelgen.curvilinear_1200x800(nt=6000)


def curvilinear_4096x2048():
    """The 4096x2048 curvilinear model (seafloor on the middle row), 1500 steps."""
    return modelgen.curvilinear_4096x2048(nt=1500)


def cpml_flat_small():
    """flat_small with CFS-PML on all four sides (boundary_type 1): a top PML band
    in the fluid instead of the free surface (Cpml::FluidSolid); 400 steps, while
    the wave is still in the grid (later the absorbed field is FP32 noise)."""
    return modelgen.make_model(120, 48, 60, npd=10, fpeak=25.0, dt=5e-4, nt=400,
                               src_x=[60], src_z=[40], boundary_type=1)


def cpml_curv_small():
    """curv_small with CFS-PML on all four sides (boundary_type 1); the grid is
    flat inside the top PML band as well."""
    return modelgen.make_model(128, 52, 64, npd=12, fpeak=25.0, dt=4e-4, nt=500,
                               src_x=[70], src_z=[44], amp=20.0, wavelength=300.0,
                               perturb=0.05, seed=3, boundary_type=1)


def solid_flat_small():
    """Solid only with a flat free surface (calc_type 0, PmlFs::SolidOnly): 120 x 100,
    10-cell PML, 25 Hz explosive source 20 rows below the surface, 400 steps."""
    return modelgen.make_solid_model(120, 100, npd=10, fpeak=25.0, dt=5e-4, nt=400,
                                     src_x=[60], src_z=[20])


def solid_curv_small():
    """Solid only with surface topography (15 m sinusoid) and 5% perturbations, 400 steps."""
    return modelgen.make_solid_model(120, 100, npd=10, fpeak=25.0, dt=5e-4, nt=400,
                                     src_x=[55], src_z=[22], amp=15.0, wavelength=300.0,
                                     perturb=0.05, seed=3)


def cpml_solid_flat_small():
    """Solid only with CFS-PML on all four sides (calc_type 0, boundary_type 1,
    Cpml::SolidOnly): 120 x 100, 10-cell PML, 25 Hz explosive source on row 40,
    record on row 30, 250 steps, while the wave is still in the grid (later the
    four-side PML has absorbed it and the final field is FP32 noise)."""
    return modelgen.make_solid_model(120, 100, npd=10, fpeak=25.0, dt=5e-4, nt=250,
                                     src_x=[60], src_z=[40], boundary_type=1)


def cpml_solid_curv_small():
    """Cpml::SolidOnly on a grid with a 15 m undulation inside (flat in both PML
    bands) and 5% perturbations, 250 steps."""
    return modelgen.make_solid_model(120, 100, npd=10, fpeak=25.0, dt=5e-4, nt=250,
                                     src_x=[55], src_z=[42], amp=15.0, wavelength=300.0,
                                     perturb=0.05, seed=3, boundary_type=1)


SOLID_CASES = ("solid_flat_small", "solid_curv_small", "cpml_solid_flat_small",
               "cpml_solid_curv_small")

# name -> (builder, receiver stride kept in the fixture, final snapshot: 0 none,
# 1 whole fields, k > 1 every k-th row and column)
CASES = {
    "flat_small": (flat_small, 1, True),
    "curv_small": (curv_small, 1, True),
    "shallow_src": (shallow_src, 1, True),
    "flat_400x400": (flat_400x400, 1, False),
    "curvilinear_1200x800": (curvilinear_1200x800, 8, 4),
    "curvilinear_4096x2048": (curvilinear_4096x2048, 8, 8),
    "cpml_flat_small": (cpml_flat_small, 1, True),
    "cpml_curv_small": (cpml_curv_small, 1, True),
    "solid_flat_small": (solid_flat_small, 1, True),
    "solid_curv_small": (solid_curv_small, 1, True),
    "cpml_solid_flat_small": (cpml_solid_flat_small, 1, True),
    "cpml_solid_curv_small": (cpml_solid_curv_small, 1, True),
}


# Cases also run through a second build of the reference with FMA contraction
# off (nvcc -fmad=false): the two builds' distance is the FP32 noise floor of
# the scheme at that length, which the CUDA path is measured against.
NOFMA_CASES = ("flat_400x400", "curvilinear_1200x800", "curvilinear_4096x2048")


def snapshot_step(keep) -> int:
    """Row/column step of a fixture's stored final snapshot (0: none)."""
    return 0 if not keep else (1 if keep is True else int(keep))


def fixture_path(name: str) -> str:
    return os.path.join(GOLDEN_DIR, name + ".npz")
