"""Tile rules (CPU): which tile shape a new shot gets."""
import pytest

from denise_b200 import _lib, synth, tune


def test_rules_pick_the_last_match_and_respect_the_class(tmp_path):
    tune.clear_rules()
    p = synth.c0_params(nx=400, ny=200)
    assert tune.tile_for(p) == (128, 8)
    tune.set_rule(8, 0, 50_000, 100_000, 64, 16)
    assert tune.tile_for(p) == (64, 16)
    tune.set_rule(8, 0, 80_000, 80_000, 256, 4)           # later and narrower: wins for this grid
    assert tune.tile_for(p) == (256, 4)
    assert tune.tile_for(p.replace(fdorder=4)) == (128, 8)  # other FDORDER: default
    assert tune.tile_for(p.replace(nx=1000)) == (128, 8)    # outside the ranges
    rules = [(8, 0, 50_000, 100_000, 64, 16), (8, 0, 80_000, 80_000, 256, 4)]
    tune.save(tmp_path / "t.json", rules)
    tune.clear_rules()
    assert tune.load(tmp_path / "t.json") == rules
    assert tune.tile_for(p) == (256, 4)
    tune.clear_rules()


@pytest.mark.parametrize("bad", [(8, 0, 0, 10, 48, 8), (8, 0, 0, 10, 128, 0), (7, 0, 0, 10, 128, 8)])
def test_bad_rules_are_rejected(bad):
    with pytest.raises(_lib.DeniseError):
        tune.set_rule(*bad)
