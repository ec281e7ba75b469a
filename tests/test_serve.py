"""Admission logic of the serving loop (CPU)."""
import numpy as np

from denise_b200 import serve, synth
from denise_b200.serve import plan_admission


def test_first_fit_in_arrival_order():
    assert plan_admission([5, 3, 9, 1], 10, 0, 8) == [0, 1, 3]
    assert plan_admission([12, 3, 1], 10, 2, 8) == [1, 2]   # the head does not fit: smaller ones pass


def test_head_of_line_is_not_starved():
    assert plan_admission([12, 3, 1], 10, 8, 8) == []        # after max_head_wait rounds nothing passes it
    assert plan_admission([12, 3, 1], 20, 8, 8) == [0, 1, 2]


def test_nothing_fits():
    assert plan_admission([30, 40], 10, 0, 8) == []
    assert plan_admission([], 10, 0, 8) == []


def test_footprint_grows_with_shots_and_storage():
    p = synth.c0_params(nx=200, ny=100, nt=400, store_snapshots=1)
    z = np.ones((200, 100), np.float32)
    sig = np.zeros((1, 400), np.float32)
    rec = (np.arange(5, 50, 5, dtype=np.int32), np.full(9, 3, np.int32))
    one = serve.Request("forward", p, (z, z, z), [(np.array([20]), np.array([2]), sig) + rec])
    two = serve.Request("forward", p, (z, z, z), [one.shots[0], one.shots[0]])
    grad = serve.Request("gradient", p, (z, z, z), [one.shots[0]])
    assert serve.footprint(two) > serve.footprint(one)
    assert serve.footprint(grad) > serve.footprint(one)
