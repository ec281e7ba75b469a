"""sharded_gradient on the GPU: two gloo ranks (independent batches on the same
device; no kernel waits on another rank) give the single-process gradient up to
the order of the float sums (partial stacks per rank, summed in float64)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracles as O
from denise_b200.shard import sharded_gradient
from test_gpu_serve import _request

pytestmark = pytest.mark.gpu


def _case():
    r = _request(0, "gradient", 72, 56, 280, 8, 0, 4, 3)
    return r.params, r.model, r.shots, r.obs


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    from datetime import timedelta

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    p, model, shots, obs = _case()
    g = sharded_gradient(p, model, shots, obs, dist, 0)
    np.save(os.path.join(out_dir, f"g{rank}.npy"), np.concatenate([x.ravel() for x in g[:3]] + [[g[3]]]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_match_one(tmp_path):
    p, model, shots, obs = _case()
    one = sharded_gradient(p, model, shots, obs, None, 0)
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    a = np.load(tmp_path / "g0.npy")
    b = np.load(tmp_path / "g1.npy")
    np.testing.assert_array_equal(a, b)
    n = p.nx * p.ny
    for k in range(3):
        assert O.rel_l2(a[k * n:(k + 1) * n], one[k].ravel()) < 1e-6
    assert abs(a[-1] - one[3]) <= 1e-12 * abs(one[3])


def test_memory_batches_give_the_same_gradient(monkeypatch):
    """A rank's shots run in batches that fit the device; forced batches of one and
    of two shots stack the same gradient bit for bit (shot order is kept) and give
    the same misfit as one batch."""
    from denise_b200 import shard

    p, model, shots, obs = _case()
    one = sharded_gradient(p, model, shots, obs, None, 0)
    assert len(shard.memory_batches(p, shots, range(len(shots)), 1, 0)) == 1   # small case: one batch
    for size in (1, 2):
        monkeypatch.setattr(shard, "memory_batches",
                            lambda params, sh, idx, store, device=0, share=0.9, size=size:
                            [list(idx)[k:k + size] for k in range(0, len(list(idx)), size)])
        got = sharded_gradient(p, model, shots, obs, None, 0)
        for a, b in zip(got[:3], one[:3]):
            np.testing.assert_array_equal(a, b)
        assert got[3] == one[3]


def _misfit_worker(rank, world, port, out_dir):
    import torch.distributed as dist
    from datetime import timedelta

    from denise_b200 import shard

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    p, model, shots, obs = _case()
    ran = []
    make = shard.make_shot
    shard.make_shot = lambda m, sh: (ran.append(next(k for k, x in enumerate(shots) if x is sh)), make(m, sh))[1]
    L2 = shard.sharded_misfit(p, model, shots, obs, range(len(shots)), dist, 0)
    np.save(os.path.join(out_dir, f"m{rank}.npy"), np.array(ran + [-1, L2]))
    dist.barrier()
    dist.destroy_process_group()


def test_step_search_misfit_two_ranks(tmp_path):
    """obj_psv.c on two ranks: each rank runs the mode-2 forwards of its own test
    shots only, and the all-reduced misfit equals the single-process one."""
    from denise_b200.shard import sharded_misfit

    p, model, shots, obs = _case()
    one = sharded_misfit(p, model, shots, obs, range(len(shots)), None, 0)
    mp.spawn(_misfit_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    r = [np.load(tmp_path / f"m{k}.npy") for k in range(2)]
    ran = [sorted(x[:-2].astype(int)) for x in r]
    assert sorted(ran[0] + ran[1]) == list(range(len(shots))) and ran[0] and ran[1]
    assert r[0][-1] == r[1][-1]
    assert abs(r[0][-1] - one) <= 1e-12 * abs(one)
