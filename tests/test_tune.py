"""Tile rules (CPU): which tile shape a new shot gets."""
import pytest

from denise_b200 import _lib, synth, tune


def test_rules_pick_the_last_match_and_respect_the_class(tmp_path):
    tune.clear_rules()
    p = synth.c0_params(nx=400, ny=200)
    big = p.replace(nx=2000, ny=600)
    assert tune.tile_for(p) == (128, 4)                   # forward default below 480 k cells
    assert tune.tile_for(big) == (128, 8)                 # forward default from 480 k cells
    assert tune.tile_for(big.replace(store_snapshots=1)) == (128, 4)   # snapshot-storing default
    tune.set_rule(8, 0, 50_000, 100_000, 64, 16)
    assert tune.tile_for(p) == (64, 16)
    tune.set_rule(8, 0, 80_000, 80_000, 256, 4)           # later and narrower: wins for this grid
    assert tune.tile_for(p) == (256, 4)
    assert tune.tile_for(p.replace(fdorder=4)) == (128, 4)  # other FDORDER: default
    assert tune.tile_for(p.replace(nx=1000)) == (128, 4)    # outside the ranges
    assert tune.default_choice(400 * 200, 0) == (128, 4, _lib.KERN_PAIRED)
    assert tune.default_choice(2000 * 600, 0) == (128, 8, _lib.KERN_PAIRED)
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


def test_kernel_variant_rules_and_snapshot_class():
    """Rules pick the register blocking too, and may hold for shots that store
    snapshots, that do not, or both."""
    tune.clear_rules()
    p = synth.c0_params(nx=400, ny=200)
    assert tune.choice_for(p) == (128, 4, _lib.KERN_PAIRED)
    tune.set_rule(8, 0, 0, 10**6, 128, 8, store=0, variant=_lib.KERN_COLUMN)
    assert tune.choice_for(p) == (128, 8, _lib.KERN_COLUMN)
    assert tune.choice_for(p.replace(store_snapshots=1)) == (128, 4, _lib.KERN_PAIRED)
    tune.set_rule(8, 0, 0, 10**6, 64, 16, store=1)               # variant -1: the default kernels
    assert tune.choice_for(p.replace(store_snapshots=1)) == (64, 16, _lib.KERN_PAIRED)
    assert tune.choice_for(p) == (128, 8, _lib.KERN_COLUMN)
    tune.clear_rules()


def test_committed_table_loads():
    """The measured table (denise_b200/tiles_b200.json) installs as rules."""
    tune.clear_rules()
    rules = tune.load(tune.TABLE)
    assert len(rules) >= 12 and all(len(r) == 10 for r in rules)
    p = synth.c0_params(nx=600, ny=300)
    assert tune.choice_for(p)[2] in (_lib.KERN_PAIRED, _lib.KERN_COLUMN)
    tune.clear_rules()
