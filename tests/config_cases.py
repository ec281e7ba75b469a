"""The benchmark workloads at their full sizes for the parity tests, and the
CPU oracle runs they are compared with (test infrastructure).

* C0: plain elastic forward, 600 x 300, NT 5000, FDORDER 8, free surface,
  120 receivers (synth.c0_case).
* C1: one shot of the batched viscoelastic workload, 2000 x 600, L = 3,
  FDORDER 8 (synth.c1_shot), shortened to NT steps.
* C2: the FWI gradient workload, 1700 x 500, DH 10 m, DT 1 ms, NT 4000,
  FDORDER 8, DTINV 2; true model = the seeded family (seed 2), starting model
  = it smoothed with sigma 25 cells, Ricker 8 Hz sources evenly spaced over 32
  positions at z = 10 m, 400 receivers at z = 20 m; observed data synthesised
  on the GPU from the true model.

The CPU functions run in spawned processes (the reference harness keeps global
state; a fresh process per run).  At C2 size one reference shot keeps 34 GB of
snapshots and one FP64 oracle shot 68 GB in host memory.
"""
import os
import time

import numpy as np

import oracles as O

C2_SHOTS = 32


def c2_case(nshots=C2_SHOTS, **kw):
    from denise_b200 import synth

    p = synth.c2_params(**kw)
    true = synth.base_model(p.nx, p.ny, p.dh, 2)
    start = tuple(synth.smoothed(x, 25.0) for x in true)
    xmax = (p.nx - 1) * p.dh
    sig = synth.ricker_source(p, 8.0)[None, :]
    ri, rj = synth.receivers_line(100.0, xmax - 100.0, 400, 20.0, p.dh)
    shots = [(np.array([synth.grid_index(200.0 + (xmax - 400.0) * k / max(nshots - 1, 1), p.dh)], np.int32),
              np.array([max(synth.grid_index(10.0, p.dh), 1)], np.int32), sig, ri, rj) for k in range(nshots)]
    return p, true, start, shots


def snapshot_bytes(p, real_bytes):
    """Host bytes of one oracle shot's snapshots (psv.c keeps 5 fields every DTINV steps)."""
    nsnap = -(-p.nt // max(p.dtinv, 1))
    return 5 * nsnap * p.nx * p.ny * real_bytes


def available_memory():
    try:
        import psutil

        return psutil.virtual_memory().available
    except ImportError:
        return os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")


def ref_forward(p, model, src, rec):
    """vx and vy sections of the reference's own forward run, and its seconds."""
    t0 = time.perf_counter()
    r = O.Reference(p, model, src, rec, mode_global=0)
    r.run(0)
    out = r.sections(0), r.sections(1)
    return out + (time.perf_counter() - t0,)


def ref_gradient_shot(p, model, shot, obs_vx, obs_vy):
    """One shot of grad_obj_psv with the reference's own code: forward with
    snapshots, calc_res (LNORM 2) of vx and vy against the observed data, the
    adjoint run and ass_gradPSV.  Returns (g_vp, g_vs, g_rho, misfit, seconds)."""
    t0 = time.perf_counter()
    r = O.Reference(p, model, shot[:3], shot[3:5], mode_global=1)
    r.run(0)
    rvx, lx = r.calc_res(obs_vx, r.sections(0))
    rvy, ly = r.calc_res(obs_vy, r.sections(1))
    r.set_residuals(rvx, rvy, None)
    r.run(1)
    g = r.ass_grad()
    return g + (lx + ly, time.perf_counter() - t0)


def fp64_gradient(p, model, shots, residuals, threads=None):
    """The FP64 restatement's stacked gradient of `shots` (double precision
    forward with double snapshots, adjoint with the given float adjoint sources,
    double accumulation), shot after shot, on `threads` OpenMP threads.
    Returns (g_vp, g_vs, g_rho, seconds)."""
    if threads:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    t0 = time.perf_counter()
    acc = [np.zeros((p.nx, p.ny), np.float64) for _ in range(3)]
    for sh, (rvx, rvy) in zip(shots, residuals):
        r = O.Restatement(p, model, sh[:3], sh[3:5], "d")
        r.forward(store=True)
        r.adjoint(rvx, rvy, None)
        for a, g in zip(acc, r.gradient()):
            a += g
        del r
    return tuple(acc) + (time.perf_counter() - t0,)
