"""Seeded synthetic models and acquisitions of the benchmark workloads, in
numpy only: no part of the CUDA library is loaded, so the reference arm of
the benchmark builds its inputs from this module alone (loaded by file path)
and runs nothing but the reference's own code.  synth.py re-exports these
functions next to the ones that use the library.

The model family (vp gradient, 6 random layer jumps, smoothed perturbations,
vs = max(vp / 1.73, 1000), rho = 310 vp^0.25, Q models) is described in
synth.py.  Arrays have the reference's file order, shape (nx, ny).
"""
import math

import numpy as np


def _smooth(noise, sigma):
    from scipy.ndimage import gaussian_filter

    return gaussian_filter(noise, sigma=sigma, mode="nearest")


def base_model(nx, ny, dh, seed, smooth_sigma=10.0):
    rng = np.random.default_rng(seed)
    z = np.arange(ny, dtype=np.float64) * dh
    zmax = max(z[-1], dh)
    vp1 = 1800.0 + 2700.0 * z / zmax
    depths = rng.uniform(0.0, zmax, 6)
    jumps = rng.uniform(-300.0, 300.0, 6)
    for d, jmp in zip(depths, jumps):
        vp1 = vp1 + np.where(z >= d, jmp, 0.0)
    vp = np.broadcast_to(vp1[None, :], (nx, ny)).copy()
    pert = _smooth(rng.standard_normal((nx, ny)), smooth_sigma)
    pert /= max(np.abs(pert).max(), 1e-30)
    vp = vp * (1.0 + 0.05 * pert)
    vs = np.maximum(vp / 1.73, 1000.0)
    rho = 310.0 * vp ** 0.25
    return vp.astype(np.float32), vs.astype(np.float32), rho.astype(np.float32)


def q_model(nx, ny, seed, smooth_sigma=10.0):
    rng = np.random.default_rng(seed + 7919)
    qp0 = rng.uniform(60.0, 120.0)
    qs0 = rng.uniform(30.0, 60.0)
    n = _smooth(rng.standard_normal((nx, ny)), smooth_sigma)
    n /= max(np.abs(n).max(), 1e-30)
    return (qp0 * (1 + 0.1 * n)).astype(np.float32), (qs0 * (1 + 0.1 * n)).astype(np.float32)


def smoothed(a, sigma):
    return _smooth(np.asarray(a, np.float64), sigma).astype(np.float32)


def add_ellipse(vp, vs, rho, dh, seed, v=5500.0):
    rng = np.random.default_rng(seed + 104729)
    nx, ny = vp.shape
    cx, cz = rng.uniform(0.3, 0.7) * nx, rng.uniform(0.4, 0.7) * ny
    ax, az = rng.uniform(0.05, 0.12) * nx, rng.uniform(0.05, 0.12) * ny
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    m = ((ii - cx) / ax) ** 2 + ((jj - cz) / az) ** 2 <= 1.0
    vp = vp.copy()
    vp[m] = v
    return vp, np.maximum(vp / 1.73, 1000.0).astype(np.float32), (310.0 * vp ** 0.25).astype(np.float32)


def iround(x):
    """fd.h:17: (int)floor(x + 0.5)."""
    return int(math.floor(x + 0.5))


def grid_index(x_m, dh):
    """Grid index of a source/receiver coordinate (sources.c, splitsrc.c:27, receiver.c:55)."""
    return iround(np.float32(x_m) / np.float32(dh))


def receivers_line(x0, x1, n, z, dh):
    xs = np.linspace(x0, x1, n)
    ri = np.array([grid_index(x, dh) for x in xs], np.int32)
    rj = np.full(n, grid_index(z, dh), np.int32)
    # receiver.c:63-83 removes receivers sharing a grid point
    keep, seen = [], set()
    for k in range(n):
        key = (int(ri[k]), int(rj[k]))
        if key not in seen:
            seen.add(key)
            keep.append(k)
    return ri[keep], rj[keep]


def ricker(nt, dt, fc, amp=1.0, tshift=0.0):
    """The Ricker wavelet of wavelet.c:38-51 (QUELLART 1) for t = nt DT, in numpy
    double arithmetic rounded to float (the library's dn_wavelet reproduces the
    reference's own rounding; this one is for inputs of the reference arm)."""
    t = np.arange(1, nt + 1, dtype=np.float32) * np.float32(dt)
    ts = 1.0 / np.float32(fc)
    tau = math.pi * (t.astype(np.float64) - 1.5 * ts - tshift) / (1.5 * ts)
    return (amp * (1.0 - 4.0 * tau * tau) * np.exp(-2.0 * tau * tau)).astype(np.float32)


def c1_acquisition(nx, ny, dh, k, nshots=64):
    """Source k of nshots evenly spaced at z = 10 m and 400 receivers at z = 20 m
    (the batched viscoelastic workload's geometry): ((src_i, src_j), (rec_i, rec_j))."""
    xmax = (nx - 1) * dh
    xs = 200.0 + (xmax - 400.0) * k / max(nshots - 1, 1)
    si = np.array([grid_index(xs, dh)], np.int32)
    sj = np.array([max(grid_index(10.0, dh), 1)], np.int32)
    return (si, sj), receivers_line(100.0, xmax - 100.0, 400, 20.0, dh)


def c1_reference_params(nx=2000, ny=600, nt=6000):
    """The batched viscoelastic workload's parameters (those of synth.c1_params:
    DH 5 m, DT 0.4 ms, FDORDER 8, Holberg MAXRELERROR 1, CPML 20 points with
    DAMPING 1500, FPML 10, npower 4, k_max_PML 1, free surface, L = 3 with
    FL 2, 8, 25 Hz, TS 1/8 s) as plain attributes, for the reference's harness."""
    from types import SimpleNamespace

    return SimpleNamespace(nx=nx, ny=ny, nt=nt, dh=5.0, dt=4e-4, fdorder=8, maxrelerror=1, free_surf=1, fw=20,
                           damping=1500.0, fpml=10.0, npower=4.0, k_max_pml=1.0, L=3, fl=(2.0, 8.0, 25.0),
                           ts=1.0 / 8.0, quelltypb=1, dtinv=1, seismo=1, eprecond=0)
