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


def _misfit_worker(rank, world, port, ntest, out_dir):
    """Each rank takes its share of the test shots (shard_of, as sharded_misfit
    does) and adds up stand-in misfits; one scalar all-reduce gives the total."""
    import torch.distributed as dist
    from datetime import timedelta

    from denise_b200.api import PsvParams
    from denise_b200.shard import allreduce_scalar, shard_of

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    p = PsvParams(nx=40, ny=30, dh=5.0, dt=1e-3, nt=100)
    test_idx = list(range(1, 2 * ntest, 2))          # TESTSHOT_START 2 .. by INCR 2 (0-based 1, 3, ...)
    mine = shard_of(p, test_idx, dist)
    total = allreduce_scalar(sum(_partial(k, (1, 1))[1] for k in mine), dist)
    np.save(os.path.join(out_dir, f"m{rank}.npy"), np.array(mine + [-1, total]))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("ntest", [5, 1])
def test_step_search_misfit_shards_test_shots(tmp_path, ntest):
    """The step-length forwards (obj_psv.c:48) run each test shot on one rank only,
    and the summed misfit is the serial one."""
    mp.spawn(_misfit_worker, args=(2, _free_port(), ntest, str(tmp_path)), nprocs=2, join=True)
    r = [np.load(tmp_path / f"m{k}.npy") for k in range(2)]
    shares = [list(x[:-2].astype(int)) for x in r]
    test_idx = list(range(1, 2 * ntest, 2))
    assert sorted(shares[0] + shares[1]) == test_idx        # every test shot on exactly one rank
    assert abs(len(shares[0]) - len(shares[1])) <= 1
    want = sum(_partial(k, (1, 1))[1] for k in test_idx)
    assert r[0][-1] == r[1][-1]
    assert abs(r[0][-1] - want) <= 1e-12 * want
