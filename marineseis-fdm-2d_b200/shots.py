"""Shot-parallel driver: independent shots (or models) sharded across ranks.

Shots never exchange data while stepping (each is its own forward run), so
the multi-GPU form is one process per GPU, each stepping its share of the
shot list on its own device, with the receiver records gathered afterwards -
no collective on the data path. The reference runs its shots one after the
other in one process (src/main.cu:94); here every shot starts from a zeroed
wavefield (the reference carries the previous shot's field over, which a
sharded run cannot reproduce).

Units of work are shared round-robin when they cost the same (the shots of
one model) and by a greedy size balance when they do not (models of uneven
size). Records travel as one padded float32 tensor per rank through
all_gather (on the device with NCCL); only a few integers of metadata per
unit go through the object collective. A gradient evaluation ends with one
all-reduce of a float32 device buffer holding the misfit and the seven
coefficient gradients, summed on each rank's device as its shots finish.
"""
from __future__ import annotations

from typing import Callable, Dict, List, Optional, Sequence

import numpy as np


def shard(nshots: int, world: int, rank: int,
          costs: Optional[Sequence[float]] = None) -> List[int]:
    """This rank's share of unit indices 0 .. nshots-1 (every unit exactly once).

    Without `costs`: round-robin. With `costs` (one per unit): the greedy
    longest-first balance - units in decreasing cost (ties by index) go one by
    one to the rank with the least total so far (ties to the lowest rank), the
    same assignment on every rank. The result is sorted."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    if costs is None:
        return list(range(rank, nshots, world))
    if len(costs) != nshots:
        raise ValueError("one cost per unit")
    load = [0.0] * world
    mine = []
    for u in sorted(range(nshots), key=lambda i: (-float(costs[i]), i)):
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += float(costs[u])
        if r == rank:
            mine.append(u)
    return sorted(mine)


def solve_on_gpu(model, shot: int, device: int = 0):
    """Default per-shot solver: a fresh wavefield on `device`, all nt steps, records."""
    import importlib
    mfdm = importlib.import_module(__package__)
    with mfdm.Solver.from_model(model, device=device) as s:
        s.set_shot(shot, reset=True)
        s.step(model.nt)
        return s.records()


def _buffer_device(dist, device: int):
    return f"cuda:{device}" if dist.get_backend() == "nccl" else "cpu"


def gather_records(local: Dict[int, dict], dist, device: int = 0) -> Dict[int, dict]:
    """Every rank's {unit: {name: float32 array}} on every rank.

    Each rank packs its arrays into one flat float32 tensor; the tensors,
    padded to the longest, go through one all_gather (device tensors with
    NCCL, host tensors with gloo). The unit ids, names and shapes go through
    all_gather_object as plain integers and strings."""
    import torch
    world = dist.get_world_size()
    meta, parts = [], []
    for unit in sorted(local):
        for name in sorted(local[unit]):
            a = np.ascontiguousarray(local[unit][name], dtype=np.float32)
            meta.append((int(unit), str(name), tuple(int(d) for d in a.shape)))
            parts.append(a.ravel())
    flat = np.concatenate(parts) if parts else np.zeros(0, np.float32)
    metas: List[Optional[list]] = [None] * world
    dist.all_gather_object(metas, meta)
    sizes = [sum(int(np.prod(sh)) for _, _, sh in m) for m in metas]
    n = max(sizes) if sizes else 0
    dev = _buffer_device(dist, device)
    buf = torch.zeros(max(n, 1), dtype=torch.float32, device=dev)
    if flat.size:
        buf[:flat.size] = torch.from_numpy(flat).to(dev)
    outs = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(outs, buf)
    merged: Dict[int, dict] = {}
    for m, t in zip(metas, outs):
        host = t.cpu().numpy()
        o = 0
        for unit, name, sh in m:
            k = int(np.prod(sh))
            merged.setdefault(unit, {})[name] = host[o:o + k].reshape(sh).copy()
            o += k
    return merged


def run_shots(model, solve: Optional[Callable] = None, dist=None, device: int = 0) -> Dict[int, dict]:
    """Runs this rank's shots (round-robin) and returns the records of every shot on every rank.

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
    return gather_records(local, dist, device)


def run_models(models: Sequence, solve: Optional[Callable] = None, dist=None,
               device: int = 0) -> Dict[int, dict]:
    """Shot 0 of each model of uneven size, the models shared by a size balance
    (cost = cells x steps), records of every model on every rank."""
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    if solve is None:
        solve = lambda m, s: solve_on_gpu(m, s, device)  # noqa: E731
    costs = [float(m.cells) * float(m.nt) for m in models]
    local = {i: solve(models[i], 0) for i in shard(len(models), world, rank, costs)}
    if dist is None:
        return local
    return gather_records(local, dist, device)


# ---- gradients over many shots -------------------------------------------------

GRAD_KEYS = ("K", "rcp_rho_f", "C11", "C13", "C33", "C55", "rcp_rho_s")


def grad_length(shapes: Dict[str, tuple]) -> int:
    return sum(int(np.prod(shapes[k])) for k in GRAD_KEYS)


def shot_gradients_on_gpu(model, shot_list, observed, device: int = 0, ckpt_every: int = 50):
    """L2 misfit and coefficient gradients of the given shots, summed, on one
    handle (the transposed operators are assembled once for all of them).
    `observed[shot]` holds the observed records {'svx', 'svz', 'fp'}. The
    gradients are summed on the device in float32: returns (misfit, flat CUDA
    tensor of the seven GRAD_KEYS arrays packed), or (0, None) without shots."""
    import importlib

    import torch
    mfdm = importlib.import_module(__package__)
    total, acc = 0.0, None
    if not shot_list:
        return total, acc
    with mfdm.Solver.from_model(model, device=device) as s:
        info = s.info()
        acc = torch.zeros((2 * info["nz_f"] + 5 * info["nz_s"]) * info["nx"], dtype=torch.float32,
                          device=f"cuda:{device}")
        for shot in shot_list:
            s.set_shot(shot, reset=True)
            rec = s.adjoint_forward(model.nt, ckpt_every)
            res = {k: rec[k].astype(np.float64) - np.asarray(observed[shot][k], np.float64)
                   for k in ("svx", "svz", "fp")}
            total += 0.5 * sum(float(np.sum(r * r)) for r in res.values())
            s.adjoint_backward_only({k: v.astype(np.float32) for k, v in res.items()})
            s.adjoint_accumulate_grad(acc)
    torch.cuda.synchronize(device)
    return total, acc


def gradient_shots(model, observed, shapes, grad: Optional[Callable] = None, dist=None,
                   device: int = 0):
    """Misfit and coefficient gradients summed over every shot of `model`.

    Each rank takes its round-robin share of the shots; `grad(model, shots)`
    returns (misfit, gradients) summed over them - gradients as a dict of
    [rows][nx] arrays or as one flat float32 tensor of the GRAD_KEYS arrays
    packed (the default, shot_gradients_on_gpu, keeps it on the device). One
    all-reduce (sum) of a float32 buffer holding the misfit (as a high and a
    low float32 part, so the sum keeps about 48 bits) and the packed gradients
    gives every rank the totals: the single collective of a gradient
    evaluation, on the device with NCCL. `shapes[key]` is the [rows][nx] shape
    of each gradient array (a rank without shots contributes zeros). Returns
    (misfit, {key: tensor [rows][nx]}), on the buffer's device.
    """
    import torch
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    if grad is None:
        grad = lambda m, sl: shot_gradients_on_gpu(m, sl, observed, device)  # noqa: E731
    j, g = grad(model, shard(len(model.src_x), world, rank))
    dev = _buffer_device(dist, device) if dist is not None else (
        g.device if isinstance(g, torch.Tensor) else "cpu")
    n = grad_length(shapes)
    buf = torch.zeros(2 + n, dtype=torch.float32, device=dev)
    hi = np.float32(j)
    buf[0] = float(hi)
    buf[1] = float(np.float32(j - float(hi)))
    if isinstance(g, torch.Tensor):
        buf[2:] = g.to(dev).reshape(-1)
    elif g is not None:
        buf[2:] = torch.from_numpy(np.concatenate(
            [np.asarray(g[k], np.float32).ravel() for k in GRAD_KEYS])).to(dev)
    if dist is not None:
        dist.all_reduce(buf, op=dist.ReduceOp.SUM)
    total = float(buf[0].item()) + float(buf[1].item())
    res, o = {}, 2
    for k in GRAD_KEYS:
        m = int(np.prod(shapes[k]))
        res[k] = buf[o:o + m].reshape(shapes[k])
        o += m
    return total, res
