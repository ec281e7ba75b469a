"""Shot sharding and the gradient sum over ranks: world-size-2 gloo process
groups on the CPU (the collective path without a GPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from denise_b200.shard import allreduce_sum, assign_shots


def test_lpt_covers_every_shot_once_and_balances():
    rng = np.random.default_rng(0)
    costs = list(rng.integers(1, 100, 37))
    for world in (1, 2, 3, 8):
        parts = assign_shots(costs, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[k] for k in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)   # LPT bound
        assert all(p == sorted(p) for p in parts)


def test_more_ranks_than_shots():
    parts = assign_shots([5, 3], 4)
    assert sorted(k for p in parts for k in p) == [0, 1]
    assert sum(1 for p in parts if not p) == 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _partial(k, shape):
    """A stand-in for shot k's gradient and misfit (deterministic per shot)."""
    rng = np.random.default_rng(100 + k)
    return [rng.standard_normal(shape).astype(np.float32) for _ in range(3)], float(rng.uniform(1, 2))


def _worker(rank, world, port, nshots, shape, out_dir):
    import torch.distributed as dist
    from datetime import timedelta

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    mine = assign_shots([1.0 + (k % 3) for k in range(nshots)], world)[rank]
    g = [np.zeros(shape, np.float64) for _ in range(3)]
    mis = 0.0
    for k in mine:
        pk, mk = _partial(k, shape)
        for a, b in zip(g, pk):
            a += b
        mis += mk
    red = allreduce_sum(g + [np.array([mis])], dist)
    np.save(os.path.join(out_dir, f"rank{rank}.npy"), np.concatenate([r.ravel() for r in red]))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("nshots", [5, 1])
def test_gradient_sum_over_two_gloo_ranks(tmp_path, nshots):
    shape = (17, 9)
    mp.spawn(_worker, args=(2, _free_port(), nshots, shape, str(tmp_path)), nprocs=2, join=True)
    want = [np.zeros(shape, np.float64) for _ in range(3)]
    mis = 0.0
    for k in range(nshots):
        pk, mk = _partial(k, shape)
        for a, b in zip(want, pk):
            a += b
        mis += mk
    flat_want = np.concatenate([w.ravel() for w in want] + [np.array([mis])])
    r0 = np.load(tmp_path / "rank0.npy")
    r1 = np.load(tmp_path / "rank1.npy")
    np.testing.assert_array_equal(r0, r1)                       # every rank holds the same sum
    np.testing.assert_allclose(r0, flat_want, rtol=1e-12, atol=1e-12)


def test_single_process_sum_is_identity():
    a = [np.ones((3, 2), np.float32), np.arange(4, dtype=np.float32)]
    out = allreduce_sum(a, None)
    np.testing.assert_array_equal(out[0], a[0])
    np.testing.assert_array_equal(out[1], a[1])
