"""Shot-parallel driver: independent shots of one model sharded across ranks.

Shots never exchange data while stepping (each is its own forward run), so
the multi-GPU form is one process per GPU, each stepping its share of the
shot list on its own device, with the receiver records gathered afterwards -
no collective on the data path. The reference runs its shots one after the
other in one process (src/main.cu:94); here every shot starts from a zeroed
wavefield (the reference carries the previous shot's field over, which a
sharded run cannot reproduce).
"""
from __future__ import annotations

from typing import Callable, Dict, List, Optional


def shard(nshots: int, world: int, rank: int) -> List[int]:
    """Round-robin share of shot indices for `rank` (every shot exactly once)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    return list(range(rank, nshots, world))


def solve_on_gpu(model, shot: int, device: int = 0):
    """Default per-shot solver: a fresh wavefield on `device`, all nt steps, records."""
    import importlib
    mfdm = importlib.import_module(__package__)
    with mfdm.Solver.from_model(model, device=device) as s:
        s.set_shot(shot, reset=True)
        s.step(model.nt)
        return s.records()


def run_shots(model, solve: Optional[Callable] = None, dist=None, device: int = 0) -> Dict[int, dict]:
    """Runs this rank's shots and returns the records of every shot on every rank.

    `dist` is torch.distributed (initialised) or None for a single process;
    `solve(model, shot)` defaults to solve_on_gpu on `device`.
    """
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    if solve is None:
        solve = lambda m, s: solve_on_gpu(m, s, device)  # noqa: E731
    local = {s: solve(model, s) for s in shard(len(model.src_x), world, rank)}
    if dist is None:
        return local
    parts: List[Optional[dict]] = [None] * world
    dist.all_gather_object(parts, local)
    merged: Dict[int, dict] = {}
    for p in parts:
        merged.update(p)
    return merged


# ---- gradients over many shots -------------------------------------------------

GRAD_KEYS = ("K", "rcp_rho_f", "C11", "C13", "C33", "C55", "rcp_rho_s")


def shot_gradients_on_gpu(model, shot_list, observed, device: int = 0, ckpt_every: int = 50):
    """L2 misfit and coefficient gradients of the given shots, summed, on one
    handle (the transposed operators are assembled once for all of them).
    `observed[shot]` holds the observed records {'svx', 'svz', 'fp'}."""
    import importlib

    import numpy as np
    mfdm = importlib.import_module(__package__)
    total, acc = 0.0, None
    if not shot_list:
        return total, acc
    with mfdm.Solver.from_model(model, device=device) as s:
        for shot in shot_list:
            s.set_shot(shot, reset=True)
            rec = s.adjoint_forward(model.nt, ckpt_every)
            res = {k: rec[k].astype(np.float64) - np.asarray(observed[shot][k], np.float64)
                   for k in ("svx", "svz", "fp")}
            total += 0.5 * sum(float(np.sum(r * r)) for r in res.values())
            g = s.adjoint_backward({k: v.astype(np.float32) for k, v in res.items()})
            acc = g if acc is None else {k: acc[k] + g[k] for k in acc}
    return total, acc


def gradient_shots(model, observed, shapes, grad: Optional[Callable] = None, dist=None,
                   device: int = 0):
    """Misfit and coefficient gradients summed over every shot of `model`.

    Each rank takes its round-robin share of the shots (`grad(model, shots)`
    returns (misfit, {key: array}) summed over them; default
    shot_gradients_on_gpu), then one all-reduce (sum) of the misfit and all
    gradient arrays packed into one buffer gives every rank the totals: the
    single collective of a gradient evaluation. `shapes[key]` is the [rows][nx]
    shape of each gradient array (a rank without shots contributes zeros).
    """
    import numpy as np
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    if grad is None:
        grad = lambda m, sl: shot_gradients_on_gpu(m, sl, observed, device)  # noqa: E731
    j, g = grad(model, shard(len(model.src_x), world, rank))
    if g is None:
        g = {k: np.zeros(shapes[k]) for k in GRAD_KEYS}
    if dist is None:
        return j, g
    import torch
    flat = np.concatenate([[j]] + [np.asarray(g[k], np.float64).ravel() for k in GRAD_KEYS])
    t = torch.from_numpy(flat)
    if dist.get_backend() == "nccl":
        t = t.to(f"cuda:{device}")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    out = t.cpu().numpy()
    res, o = {}, 1
    for k in GRAD_KEYS:
        n = int(np.prod(shapes[k]))
        res[k] = out[o:o + n].reshape(shapes[k])
        o += n
    return float(out[0]), res
