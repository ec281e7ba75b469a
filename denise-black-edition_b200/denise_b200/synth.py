"""Seeded synthetic inputs of the benchmark workloads.

No public dataset is named for this path; the reference's Marmousi-II inputs
are not available.  Every model here is drawn from one seeded family:

* vp(z) = 1800 + 2700 z / z_max, plus 6 layer boundaries at depths uniform in
  (0, z_max) that each add a jump uniform in (-300, 300) m/s below them, plus
  Gaussian-smoothed (sigma 10 cells) N(0, 1) noise normalised to max |.| = 1
  and scaled by 0.05 vp;
* vs = max(vp / 1.73, 1000), rho = 310 vp^0.25 (Gardner);
* viscoelastic runs add Qp ~ U(60, 120), Qs ~ U(30, 60) per model, times
  (1 + 0.1 smoothed noise).

Arrays have the reference's file order, shape (nx, ny).
"""
import math

import numpy as np

from .api import PsvParams, wavelet
from .modelgen import (_smooth, add_ellipse, base_model, c1_acquisition, grid_index, iround, q_model,  # noqa: F401
                       receivers_line, smoothed)


def ricker_source(p: PsvParams, fc, amp=1.0, tshift=0.0):
    return wavelet(1, p.nt, p.dt, tshift, fc, amp)


# ---------------------------------------------------------------------------
# the benchmark configurations
# ---------------------------------------------------------------------------
def c0_params(**kw):
    """Plain elastic forward: 600 x 300, DH 5 m, DT 0.4 ms, NT 5000, FDORDER 8, FW 20, free surface."""
    base = dict(nx=600, ny=300, dh=5.0, dt=4e-4, nt=5000, fdorder=8, maxrelerror=1, free_surf=1, fw=20,
                damping=1500.0, fpml=10.0, npower=4.0, k_max_pml=1.0, ts=0.1)
    base.update(kw)
    return PsvParams(**base)


def c0_case(seed=0, **kw):
    p = c0_params(**kw)
    vp, vs, rho = base_model(p.nx, p.ny, p.dh, seed)
    sig = ricker_source(p, 10.0)[None, :]
    si = np.array([grid_index(1500.0 * p.nx / 600.0, p.dh)], np.int32)
    sj = np.array([max(grid_index(10.0, p.dh), 1)], np.int32)
    ri, rj = receivers_line(100.0 * p.nx / 600.0, 2900.0 * p.nx / 600.0, 120, 20.0, p.dh)
    return p, (vp, vs, rho), (si, sj, sig), (ri, rj)


C1_FL = (2.0, 8.0, 25.0)   # relaxation frequencies for L = 3 (not given by the workload; chosen here)


def c1_params(**kw):
    """Batched viscoelastic: 2000 x 600, DH 5, DT 0.4 ms, NT 6000, FDORDER 8, L 3."""
    base = dict(nx=2000, ny=600, dh=5.0, dt=4e-4, nt=6000, fdorder=8, maxrelerror=1, free_surf=1, fw=20,
                damping=1500.0, fpml=10.0, npower=4.0, k_max_pml=1.0, L=3, fl=C1_FL, ts=1.0 / 8.0)
    base.update(kw)
    return PsvParams(**base)


def c1_shot(p: PsvParams, k, nshots=64, seed=None):
    """Shot k of the batched workload: its own model (seed k+1), source k of nshots."""
    seed = k + 1 if seed is None else seed
    vp, vs, rho = base_model(p.nx, p.ny, p.dh, seed)
    qp, qs = q_model(p.nx, p.ny, seed)
    (si, sj), (ri, rj) = c1_acquisition(p.nx, p.ny, p.dh, k, nshots)
    sig = ricker_source(p, 8.0)[None, :]
    return (vp, vs, rho, qp, qs), (si, sj, sig), (ri, rj)


def c2_params(**kw):
    """FWI gradient: 1700 x 500, DH 10, DT 1 ms, NT 4000, FDORDER 8, DTINV 2."""
    base = dict(nx=1700, ny=500, dh=10.0, dt=1e-3, nt=4000, fdorder=8, maxrelerror=1, free_surf=1, fw=20,
                damping=1500.0, fpml=10.0, npower=4.0, k_max_pml=1.0, ts=1.0 / 8.0, dtinv=2, quelltypb=1,
                store_snapshots=1)
    base.update(kw)
    return PsvParams(**base)


# ---------------------------------------------------------------------------
# the serving workload: a seeded stream of requests of mixed size and kind
# ---------------------------------------------------------------------------
SERVE_MIX = (("forward", 0, 0.7), ("forward", 3, 0.2), ("gradient", 0, 0.1))   # kind, L, share


def serve_requests(n, seed=3, scale=1.0, snap_budget=16e9, first=0, last=None):
    """n requests: 70 % elastic forward, 20 % viscoelastic (L = 3) forward, 10 %
    elastic FWI gradients; NX in U[300, 3000], NZ in U[150, 1000], DH in U[5, 10],
    NT in U[2000, 8000], FDORDER in {4, 8, 12}, 1-4 shots and 50-500 receivers
    per request, the model of request k from seed 1000 + k, DT = 0.9 of the CFL
    limit (checkfd_ssg_elastic.c:89).  `scale` shrinks NX, NZ and NT for quick
    runs.  Gradient requests store FP16 snapshots every DTINV steps, DTINV the
    smallest even interval that keeps one shot's snapshots under snap_budget
    bytes; their observed data are zero traces.  Returns (kind, params, model,
    shots, obs) tuples; shots are (src_i, src_j, signals, rec_i, rec_j).
    first, last: build only requests first .. last - 1 of the n-request stream
    (the same requests as in the whole stream), e.g. to build it in parallel."""
    from .api import cfl_limit

    rng = np.random.default_rng(seed)
    kinds = rng.choice(len(SERVE_MIX), size=n, p=[m[2] for m in SERVE_MIX])
    out = []
    last = n if last is None else min(last, n)
    for k in range(n):
        kind, L, _ = SERVE_MIX[kinds[k]]
        nx = max(60, int(rng.integers(300, 3001) * scale))
        ny = max(40, int(rng.integers(150, 1001) * scale))
        dh = float(rng.uniform(5.0, 10.0))
        nt = max(200, int(rng.integers(2000, 8001) * scale))
        fdorder = int(rng.choice([4, 8, 12]))
        nshots = int(rng.integers(1, 5))
        nrec = int(rng.integers(50, 501))
        if not first <= k < last:
            continue
        vp, vs, rho = base_model(nx, ny, dh, 1000 + k, smooth_sigma=4.0)
        model = (vp, vs, rho)
        kw = dict(nx=nx, ny=ny, dh=dh, nt=nt, fdorder=fdorder, maxrelerror=1, free_surf=1, fw=20,
                  damping=1500.0, fpml=10.0, npower=4.0, k_max_pml=1.0, L=L, fl=C1_FL[:L], ts=1.0 / 8.0)
        if L:
            model = model + q_model(nx, ny, 1000 + k, smooth_sigma=4.0)
        if kind == "gradient":
            per_snap = 5 * 2 * nx * ny
            dtinv = 2
            while nt / dtinv * per_snap > snap_budget:
                dtinv += 2
            kw.update(store_snapshots=1, dtinv=dtinv, snap_precision=1)
        p = PsvParams(dt=1e-3, **kw)
        dtstab, _ = cfl_limit(p, float(vp.max()))
        p = p.replace(dt=float(np.float32(0.9 * dtstab)))
        sig = wavelet(1, nt, p.dt, 0.0, 8.0, 1.0)[None, :]
        xmax = (nx - 1) * dh
        nr = min(nrec, nx - 2 * 20 - 2)
        ri, rj = receivers_line(min(100.0, 0.1 * xmax), xmax - min(100.0, 0.1 * xmax), nr, 20.0, dh)
        rj = np.maximum(rj, 1)
        shots = []
        for s in range(nshots):
            xs = 0.2 * xmax + 0.6 * xmax * s / max(nshots - 1, 1)
            shots.append((np.array([max(1, grid_index(xs, dh))], np.int32),
                          np.array([max(1, grid_index(10.0, dh))], np.int32), sig, ri, rj))
        obs = None
        if kind == "gradient":
            z = np.zeros((len(ri), nt), np.float32)
            obs = [(z, z) for _ in range(nshots)]
        out.append((kind, p, model, shots, obs))
    return out
