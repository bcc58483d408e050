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
