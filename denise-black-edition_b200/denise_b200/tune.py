"""Autotuner of the stencil tiles.

For a class of runs (FDORDER, L and a grid size) it times the time step of a
seeded batch of shots for each candidate tile shape (columns x rows of a CTA)
with per-kernel CUDA events (dn_profile_steps), and installs the fastest as a
rule for new shots of that class (dn_set_tile_shape).  Rules can be saved to
and loaded from a JSON file, so a tuned table can be reused without tuning.
Results do not depend on the tile shape; only the speed does.
"""
import ctypes
import json

import numpy as np

from . import _lib
from ._lib import check, lib

CANDIDATES = ((64, 8), (128, 4), (128, 8), (128, 16), (256, 8))


def set_rule(fdorder, L, cells_min, cells_max, bx, zch):
    check(lib.dn_set_tile_shape(int(fdorder), int(L), int(cells_min), int(cells_max), int(bx), int(zch)))


def clear_rules():
    check(lib.dn_clear_tile_shapes())


def tile_for(params):
    bx, zch = ctypes.c_int(), ctypes.c_int()
    p = params.to_c()
    check(lib.dn_get_tile_shape(ctypes.byref(p), ctypes.byref(bx), ctypes.byref(zch)))
    return bx.value, zch.value


def autotune(params, nshots=8, candidates=CANDIDATES, steps=20, device=0, span=2.0, apply=True):
    """Times each candidate on `nshots` seeded shots of `params`' grid and returns
    (best, {candidate: ms per step}); with apply, installs best for grids of
    nx*ny within a factor `span` of this one."""
    from . import api as dn
    from . import synth

    p = params.replace(nt=max(steps + 5, 10), store_snapshots=0)
    models = []
    for k in range(nshots):
        vp, vs, rho = synth.base_model(p.nx, p.ny, p.dh, 500 + k, smooth_sigma=4.0)
        extra = synth.q_model(p.nx, p.ny, 500 + k, smooth_sigma=4.0) if p.L else (None, None)
        models.append(dn.Model(p, vp, vs, rho, *extra, device=device))
    sig = np.zeros((1, p.nt), np.float32)
    sig[0, 2] = 1.0
    ri = np.arange(2, p.nx, max(1, p.nx // 64), dtype=np.int32)
    rj = np.full(len(ri), 2, np.int32)
    cells = p.nx * p.ny
    times = {}
    for bx, zch in candidates:
        set_rule(p.fdorder, p.L, cells, cells, bx, zch)
        shots = [dn.Shot(m, [p.nx // 2], [2], sig, ri, rj) for m in models]
        dn.profile_steps(shots, _lib.MODE_FORWARD, nsteps=3)
        prof = dn.profile_steps(shots, _lib.MODE_FORWARD, nsteps=steps)
        times[(bx, zch)] = float(sum(prof.values()))
        for s in shots:
            s.close()
    for m in models:
        m.close()
    best = min(times, key=times.get)
    if apply:
        set_rule(p.fdorder, p.L, int(cells / span), int(cells * span), *best)
    return best, times


def save(path, rules):
    """rules: iterable of (fdorder, L, cells_min, cells_max, bx, zch)."""
    with open(path, "w") as f:
        json.dump([list(r) for r in rules], f, indent=1)


def load(path):
    with open(path) as f:
        rules = [tuple(r) for r in json.load(f)]
    for r in rules:
        set_rule(*r)
    return rules
