"""Multi-rank shot sharding on CPU: world size 2, gloo backend, a fake per-shot solver."""
import importlib
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

shots = importlib.import_module("marineseis-fdm-2d_b200.shots")


def test_balanced_shard_covers_every_unit_once_and_balances():
    rng = np.random.default_rng(0)
    for n in (0, 1, 7, 32):
        costs = rng.integers(1, 100, n).astype(float)
        for world in (1, 2, 3, 8):
            parts = [shots.shard(n, world, r, costs) for r in range(world)]
            assert sorted(u for p in parts for u in p) == list(range(n))
            loads = [sum(costs[u] for u in p) for p in parts]
            if n:  # greedy longest-first: no rank exceeds the mean by more than the largest unit
                assert max(loads) <= sum(costs) / world + max(costs)
    # the big unit alone on one rank, the small ones on the other
    assert shots.shard(4, 2, 0, [10, 1, 1, 1]) == [0]
    assert shots.shard(4, 2, 1, [10, 1, 1, 1]) == [1, 2, 3]


def test_shard_covers_every_shot_once():
    for n in (0, 1, 5, 64):
        for world in (1, 2, 3, 8):
            got = sorted(s for r in range(world) for s in shots.shard(n, world, r))
            assert got == list(range(n))
    with pytest.raises(ValueError):
        shots.shard(4, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _Model:
    def __init__(self, n):
        self.src_x = list(range(10, 10 + n))
        self.nt = 3


def _fake_solve(model, shot):
    return {"fp": np.full((2, 4), float(shot) + 100.0 * dist.get_rank(), dtype=np.float32)}


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = shots.run_shots(_Model(5), solve=_fake_solve, dist=dist)
        np.save(os.path.join(out, f"rank{rank}.npy"),
                np.array([[s, float(res[s]["fp"][0, 0])] for s in sorted(res)]))
    finally:
        dist.destroy_process_group()


def _uneven_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        class M:
            def __init__(self, i):
                self.cells, self.nt, self.i = 100 * (i + 1), 10, i

        def solve(m, shot):  # records of a model-dependent shape
            return {"svz": np.full((3, m.i + 2), m.i + 0.5, np.float32),
                    "fp": np.arange(m.i + 1, dtype=np.float32) + 100 * dist.get_rank()}

        res = shots.run_models([M(i) for i in range(5)], solve=solve, dist=dist)
        np.save(os.path.join(out, f"models{rank}.npy"),
                np.array([[i, res[i]["svz"].shape[1], float(res[i]["svz"][0, 0]),
                           float(res[i]["fp"][-1])] for i in sorted(res)]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_run_uneven_models_balanced(tmp_path):
    port = _free_port()
    mp.spawn(_uneven_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    a = np.load(tmp_path / "models0.npy")
    b = np.load(tmp_path / "models1.npy")
    assert np.array_equal(a, b)
    assert a[:, 0].tolist() == [0, 1, 2, 3, 4]
    assert a[:, 1].tolist() == [2, 3, 4, 5, 6] and a[:, 2].tolist() == [0.5, 1.5, 2.5, 3.5, 4.5]
    # costs 100..500: rank 0 takes 500, 200, 100 (800), rank 1 takes 400, 300 (700)
    owner = {i: int((a[i, 3] - i) // 100) for i in range(5)}
    assert owner == {0: 0, 1: 0, 2: 1, 3: 1, 4: 0}


def test_two_ranks_gather_all_records(tmp_path):
    port = _free_port()
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    a = np.load(tmp_path / "rank0.npy")
    b = np.load(tmp_path / "rank1.npy")
    assert np.array_equal(a, b)  # every rank sees every shot
    assert a[:, 0].tolist() == [0, 1, 2, 3, 4]
    # shot s was solved by rank s % 2 (round robin)
    assert a[:, 1].tolist() == [s + 100.0 * (s % 2) for s in range(5)]


SHAPES = {"K": (2, 3), "rcp_rho_f": (2, 3), "C11": (4, 3), "C13": (4, 3), "C33": (4, 3),
          "C55": (4, 3), "rcp_rho_s": (4, 3)}


def _fake_grad(model, shot_list):
    if not shot_list:
        return 0.0, None
    g = {k: sum(np.full(v, float(s + 1)) for s in shot_list) for k, v in SHAPES.items()}
    return float(sum(10 * (s + 1) for s in shot_list)), g


def _grad_worker(rank, world, port, out, nshots):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        j, g = shots.gradient_shots(_Model(nshots), {}, SHAPES, grad=_fake_grad, dist=dist)
        np.save(os.path.join(out, f"grad{rank}.npy"),
                np.concatenate([[j], g["C55"].numpy().ravel(), g["K"].numpy().ravel()]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nshots", [5, 1])
def test_two_ranks_sum_gradients(tmp_path, nshots):
    port = _free_port()
    mp.spawn(_grad_worker, args=(2, port, str(tmp_path), nshots), nprocs=2, join=True)
    a = np.load(tmp_path / "grad0.npy")
    b = np.load(tmp_path / "grad1.npy")
    assert np.array_equal(a, b)  # every rank holds the totals
    total = sum(range(1, nshots + 1))
    assert a[0] == 10 * total
    assert np.all(a[1:] == total)  # each shot once (one rank may have no shot)
