"""Material parameterisation of the adjoint gradients.

The library differentiates with respect to the seven coefficient arrays it
steps with (``mfdm_coef_grad``: K and 1/rho of the fluid; C11, C13, C33, C55 and
1/rho of the solid). For an isotropic model these follow from vp, vs and rho:
C11 = C33 = rho vp^2, C13 = rho (vp^2 - 2 vs^2), C55 = rho vs^2, K = rho_f vp_f^2,
and this module applies the chain rule. ``SeismicRecords`` wraps a forward run
and its adjoint as a torch.autograd.Function.
"""
from __future__ import annotations

import copy
from typing import Dict

import numpy as np


def params_of(model) -> Dict[str, np.ndarray]:
    """(vp, vs, rho) of the solid and (vp_f, rho_f) of the fluid from the
    model's coefficient arrays (float64)."""
    rs = np.asarray(model.solid["rho"], np.float64)
    rf = np.asarray(model.fluid["rho"], np.float64)
    return {"vp": np.sqrt(np.asarray(model.solid["C11"], np.float64) / rs),
            "vs": np.sqrt(np.asarray(model.solid["C55"], np.float64) / rs),
            "rho": rs,
            "vp_f": np.sqrt(np.asarray(model.fluid["K"], np.float64) / rf),
            "rho_f": rf}


def with_params(model, p: Dict[str, np.ndarray]):
    """Copy of ``model`` with isotropic coefficients built from ``p``."""
    m = copy.deepcopy(model)
    vp, vs, rho = (np.asarray(p[k], np.float64) for k in ("vp", "vs", "rho"))
    mu = rho * vs ** 2
    lam = rho * (vp ** 2 - 2.0 * vs ** 2)
    m.solid = {"C11": lam + 2 * mu, "C13": lam, "C33": lam + 2 * mu, "C55": mu, "rho": rho.copy()}
    rf = np.asarray(p["rho_f"], np.float64)
    m.fluid = {"K": rf * np.asarray(p["vp_f"], np.float64) ** 2, "rho": rf.copy()}
    return m


def chain_rule(g: Dict[str, np.ndarray], p: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
    """Coefficient gradients (mfdm_coef_grad) to gradients with respect to
    vp, vs, rho (solid) and vp_f, rho_f (fluid)."""
    vp, vs, rho = p["vp"], p["vs"], p["rho"]
    gsum = g["C11"] + g["C33"] + g["C13"]
    out = {"vp": 2 * rho * vp * gsum,
           "vs": 2 * rho * vs * (g["C55"] - 2 * g["C13"]),
           "rho": vp ** 2 * gsum - 2 * vs ** 2 * g["C13"] + vs ** 2 * g["C55"]
                  - g["rcp_rho_s"] / rho ** 2}
    vpf, rf = p["vp_f"], p["rho_f"]
    out["vp_f"] = 2 * rf * vpf * g["K"]
    out["rho_f"] = vpf ** 2 * g["K"] - g["rcp_rho_f"] / rf ** 2
    return out


def _autograd_function():
    import torch

    class SeismicRecords(torch.autograd.Function):
        """records = F(vp, vs, rho, vp_f, rho_f): one shot of ``model`` (its
        geometry, metric and source) run for ``nsteps`` steps on ``solver``;
        records are [samples][3][nx] (svx, svz, fp). backward() runs the
        adjoint (checkpoint every ``ckpt_every`` steps)."""

        @staticmethod
        def forward(ctx, vp, vs, rho, vp_f, rho_f, solver, model, nsteps, ckpt_every=50):
            p = {"vp": vp, "vs": vs, "rho": rho, "vp_f": vp_f, "rho_f": rho_f}
            p = {k: v.detach().cpu().double().numpy() for k, v in p.items()}
            solver.load_model(with_params(model, p))
            rec = solver.adjoint_forward(int(nsteps), int(ckpt_every))
            ctx.solver, ctx.p = solver, p
            out = np.stack([rec["svx"], rec["svz"], rec["fp"]], axis=1)
            return torch.from_numpy(out).to(vp.device, torch.float64)

        @staticmethod
        def backward(ctx, grad_rec):
            r = grad_rec.detach().cpu().float().numpy()
            g = ctx.solver.adjoint_backward({"svx": r[:, 0], "svz": r[:, 1], "fp": r[:, 2]})
            gp = chain_rule(g, ctx.p)
            dev = grad_rec.device
            t = [torch.from_numpy(gp[k]).to(dev) for k in ("vp", "vs", "rho", "vp_f", "rho_f")]
            return (*t, None, None, None, None)

    return SeismicRecords


_cached = {}


def __getattr__(name):
    if name == "SeismicRecords":
        if name not in _cached:
            _cached[name] = _autograd_function()
        return _cached[name]
    raise AttributeError(name)
