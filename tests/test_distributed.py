"""The batched configuration across ranks, on CPU: two `gloo` processes split a batch of systems
(baas_b200.distributed), each solves its share -- here with the oracle's PCG, standing in for a
GPU's batched launch -- and one gather brings every system's result to rank 0, which must equal a
single-process solve of the whole batch."""
import os
import socket

import numpy as np
import pytest

from baas_b200 import gen
from baas_b200.distributed import solve_sharded, split_systems


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _systems():
    return [gen.vardiff2d(k, seed=10 + q) for q, k in enumerate((12, 20, 9, 16, 24, 11, 14))]


def _solve_one(S, q):
    from oracle.oracle import Port

    x, it, rel = Port.pcg(S, gen.uniform_rhs(S.n, 100 + q), tol=1e-10, maxiter=2000)
    return {"x": x, "iterations": it, "relres": rel}


def _rank(rank, world, port, out_path):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        systems = _systems()
        got = solve_sharded(systems, lambda idx: {q: _solve_one(systems[q], q) for q in idx}, rank, world)
        if rank == 0:
            np.save(out_path, np.array([got], dtype=object), allow_pickle=True)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_split_is_a_balanced_partition():
    sizes = [S.n for S in _systems()]
    for world in (1, 2, 3, 8):
        parts = split_systems(sizes, world)
        assert sorted(q for p in parts for q in p) == list(range(len(sizes)))
        loads = [sum(sizes[q] for q in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)
    assert split_systems(sizes, 2) == split_systems(list(sizes), 2)  # deterministic


def test_two_gloo_ranks_match_one_process(tmp_path):
    import torch.multiprocessing as mp

    out = tmp_path / "gathered.npy"
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, str(out)), nprocs=2, join=True, start_method="spawn")
    got = np.load(out, allow_pickle=True)[0]
    systems = _systems()
    assert sorted(got) == list(range(len(systems)))
    for q, S in enumerate(systems):
        want = _solve_one(S, q)
        assert got[q]["iterations"] == want["iterations"]
        assert np.array_equal(got[q]["x"], want["x"])


@pytest.mark.parametrize("world", [1])
def test_single_rank_needs_no_process_group(world):
    systems = _systems()[:3]
    got = solve_sharded(systems, lambda idx: {q: q * 10 for q in idx}, 0, world)
    assert got == {0: 0, 1: 10, 2: 20}
