"""Gradient conditioning on the CPU: the oracle (oracle/precond_oracle.py)
pinned against the reference's own precond_PSV, taper_grad_shot and
smooth_grad, and the library's host-side taper coefficients and argument
checks against the oracle (no device needed for either)."""
import os
import sys

import numpy as np
import pytest

import oracles as O

sys.path.insert(0, os.path.join(O.ROOT, "oracle"))
import precond_oracle as po  # noqa: E402

from denise_b200 import DeniseError  # noqa: E402
from denise_b200.precond import PrecondConfig, PrecondPlan, taper_coefficients  # noqa: E402

needs_ref = pytest.mark.skipif(not O.reference_available(), reason="reference build not present")

NX, NY, DH = 60, 40, 5.0
# sources: one at x = 0 (its FILTSIZE box reaches columns -2..2, which the
# reference's zeroing loop maps into the row above), one on the right edge,
# one below the free surface, one at the left edge
SRCS = [(0.0, 40.0), (150.0, 30.0), (297.0, 5.0), (3.0, 60.0)]
RECS = [(5, 4), (20, 4), (60, 10), (1, 1)]
GRADT = (3, 9, 45, 55)


def bits_equal(a, b):
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    same = (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))
    return bool(same.all()), int((~same).sum())


def grads(seed=1):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((NY, NX)).astype(np.float32) for _ in range(3)]


def cfg_dict(sw, shape, radius=12.0, filtsize=2, files=None):
    return dict(taper_vert=sw[0], taper_hor=sw[1], taper_sources=sw[2], taper_file=sw[3], gradt=GRADT, exp_hor=1.5,
                srtshape=shape, srtradius=radius, filtsize=filtsize, srcs=SRCS, recs=RECS, file=files)


def write_taper_files(d, files):
    for a, sfx in zip(files, ("", "_u", "_rho")):
        np.ascontiguousarray(a.T, np.float32).tofile(os.path.join(d, f"tp{sfx}.bin"))


@needs_ref
@pytest.mark.parametrize("sw", [(1, 0, 0, 0), (0, 1, 0, 0), (0, 0, 1, 0), (0, 0, 0, 1), (1, 1, 1, 1)])
@pytest.mark.parametrize("shape", [1, 2])
def test_oracle_tapers_match_reference(tmp_path, sw, shape):
    gs = grads()
    rng = np.random.default_rng(7)
    files = [rng.random((NY, NX)).astype(np.float32) for _ in range(3)]
    write_taper_files(str(tmp_path), files)
    ref = O.run_isolated(O.ref_precond, str(tmp_path), NX, NY, DH, np.array(sw, np.int32), np.array(GRADT, np.int32),
                         1.5, shape, 12.0, 2, SRCS, RECS, gs)
    for c in range(3):
        o = po.precond_tapers(gs[c], NX, NY, DH, dict(cfg_dict(sw, shape, files=files), cls=c))
        assert bits_equal(o, ref[c]) == (True, 0), (sw, shape, c)


@needs_ref
def test_oracle_zeroed_box_wraps_like_the_reference(tmp_path):
    """The source at x = 0 with FILTSIZE 3 zeroes cells at the right end of the rows above it."""
    cells = po.zeroed_cells(NX, NY, [po.source_cell(0.0, 40.0, DH)], 3, True)
    assert any(c == NX for _, c in cells)
    gs = grads(3)
    ref = O.run_isolated(O.ref_precond, str(tmp_path), NX, NY, DH, np.array((0, 0, 1, 0), np.int32),
                         np.array(GRADT, np.int32), 1.5, 1, 12.0, 3, SRCS, RECS, gs)
    o = po.precond_tapers(gs[0], NX, NY, DH, dict(cfg_dict((0, 0, 1, 0), 1, filtsize=3), cls=0))
    assert bits_equal(o, ref[0]) == (True, 0)
    assert ref[0][7, NX - 1] == 0.0 and gs[0][7, NX - 1] != 0.0


@needs_ref
@pytest.mark.parametrize("ishot", [1, 2, 3, 4])
def test_oracle_shot_taper_matches_reference(tmp_path, ishot):
    g = grads(2)[0]
    ref = O.run_isolated(O.ref_taper_shot, str(tmp_path), NX, NY, DH, 1, 12.0, 2, SRCS, ishot, g)
    o = po.shot_taper_apply(g, NX, NY, DH, SRCS[ishot - 1], 1, 12.0, 2)
    assert bits_equal(o, ref) == (True, 0)


@needs_ref
@pytest.mark.parametrize("sf,a,b", [(2, 2.0, 3.0), (2, 0.7, 0.0), (3, 1.0, 0.0), (3, 0.3, 0.0), (4, 1.0, 0.8),
                                    (4, 0.5, 0.5)])
def test_oracle_smoothing_matches_reference(tmp_path, sf, a, b):
    g = grads(4)[1]
    vel = (1500 + 1000 * np.random.default_rng(5).random((NY, NX))).astype(np.float32)
    ref = O.run_isolated(O.ref_smooth_grad, str(tmp_path), NX, NY, DH, sf, a, b, 10.0, 400.0, vel, g)
    o = po.smooth_grad(g, sf, a, b, 10.0, 400.0, DH, vel)
    assert bits_equal(o, ref) == (True, 0)


def config(sw, shape=1, **kw):
    return PrecondConfig(taper_vert=sw[0], taper_hor=sw[1], taper_sources=sw[2], taper_file=sw[3], gradt=GRADT,
                         exp_taper_grad_hor=1.5, srtshape=shape, srtradius=12.0, filtsize=2, sources=SRCS,
                         receivers=RECS, **kw)


@pytest.mark.parametrize("shape", [1, 2])
@pytest.mark.parametrize("gradt", [GRADT, (5, 9, 0, 0), (0, 0, 30, 30), (9, 3, 45, 55)])
def test_host_taper_coefficients_match_oracle(shape, gradt):
    c = config((1, 1, 1, 0), shape)
    c.gradt = gradt
    want = {1: po.taper_vertical(NX, NY, gradt), 2: po.taper_horizontal(NX, NY, DH, gradt, 1.5),
            3: po.taper_sources(NX, NY, DH, SRCS, shape, 12.0)}
    for sws, w in want.items():
        got = taper_coefficients(NX, NY, DH, c, sws)
        assert bits_equal(got.T, w) == (True, 0), sws


def test_argument_errors():
    with pytest.raises(DeniseError, match="DN_ENOTSUP"):
        PrecondPlan(NX, NY, DH, PrecondConfig(spatfilter=1))
    with pytest.raises(DeniseError, match="DN_EINVAL"):
        PrecondPlan(1, NY, DH, PrecondConfig(taper_vert=1, gradt=(9, 3, 45, 55)))
    with pytest.raises(DeniseError, match="DN_EINVAL"):
        PrecondPlan(NX, NY, DH, PrecondConfig(taper_sources=1, srtshape=3, srtradius=10.0, sources=SRCS))
    with pytest.raises(DeniseError, match="DN_EINVAL"):
        PrecondPlan(NX, NY, DH, PrecondConfig(spatfilter=3, fc_end=0.0))
    with pytest.raises(DeniseError, match="DN_EINVAL"):
        PrecondPlan(NX, NY, DH, PrecondConfig(taper_file=1))
