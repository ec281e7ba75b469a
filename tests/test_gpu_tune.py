"""The autotuner on the GPU, and results that do not depend on the tile shape."""
import numpy as np
import pytest

import denise_b200 as dn
from denise_b200 import tune

from test_gpu_parity import gpu_shot, small_case

pytestmark = pytest.mark.gpu


def test_autotune_installs_the_fastest_candidate():
    tune.clear_rules()
    p, *_ = small_case(nx=300, ny=120)
    best, times = tune.autotune(p, nshots=2, candidates=((64, 8), (128, 8), (128, 16)), steps=10)
    assert best == min(times, key=times.get) and all(t > 0 for t in times.values())
    assert tune.tile_for(p) == best
    tune.clear_rules()


def test_sections_do_not_depend_on_the_tile_shape():
    tune.clear_rules()
    p, model, src, rec = small_case(L=3, nx=150, ny=70, store_snapshots=1)
    out = []
    for bx, zch in ((128, 8), (64, 16), (256, 4)):
        tune.set_rule(p.fdorder, p.L, 0, 10**9, bx, zch)
        m, s = gpu_shot(p, model, src, rec)
        dn.run([s])
        out.append((s.sections(dn.SEC_VX), s.field(2)))
        s.close()
        m.close()
    tune.clear_rules()
    for a, b in out[1:]:
        np.testing.assert_array_equal(a, out[0][0])
        np.testing.assert_array_equal(b, out[0][1])


@pytest.mark.parametrize("nshots", [1, 3])
def test_batch_chosen_rows_change_nothing_but_speed(monkeypatch, nshots):
    """Shots without snapshots or rules take the tile rows their batch's total cells
    call for (one row for a few small grids); with DN_AUTO_ROWS=0 they keep their
    own tiles.  Sections and final fields are the same either way, and the one-row
    batch takes fewer device milliseconds than the four-row one."""
    tune.clear_rules()
    cases = [small_case(L=L, nx=300, ny=120, nt=400, seed=3 + k) for k, L in enumerate((0, 0, 0)[:nshots])]
    res = {}
    for auto in ("1", "0"):
        monkeypatch.setenv("DN_AUTO_ROWS", auto)
        pairs = [gpu_shot(*c) for c in cases]
        shots = [s for _, s in pairs]
        dn.run(shots)
        ms = min(dn.run(shots) or dn.last_run_stats()[0] for _ in range(3))
        res[auto] = ([(s.sections(dn.SEC_VY), s.field(2)) for s in shots], ms)
        for m, s in pairs:
            s.close()
            m.close()
    for (a, fa), (b, fb) in zip(res["1"][0], res["0"][0]):
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(fa, fb)
    assert res["1"][1] < res["0"][1], (res["1"][1], res["0"][1])
