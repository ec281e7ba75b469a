"""ORACLE / TEST INFRASTRUCTURE - never part of the product.

numpy restatement of the reference's gradient conditioning after shot
stacking (FWI_PSV.c:628-634): smooth_grad (src/smooth_grad.c) followed by
precond_PSV (src/PSV/precond_PSV.c), and of the per-shot circular taper
taper_grad_shot (src/taper_grad_shot.c, grad_obj_psv.c:242-250).

Every float operation is spelled out in float32 and every term the C source
promotes to double is evaluated in Python floats (IEEE double), with the
transcendental functions (exp, erf, log, pow) taken from the C library through
the math module, as the reference's C calls them, so the results are the
reference's bits.  Gradients are [NY][NX] float32 arrays indexed [j-1][i-1]
(row j = depth, column i = x, the reference's waveconv[j][i]).

Pinned against the reference's own functions compiled by oracle/Makefile
(tests/test_precond.py, through oracle/ref_harness.c).
"""
import math

import numpy as np

f32 = np.float32


def cdiv(a, b):
    """C double division a / b (IEEE: x/0 is +-inf, 0/0 is NaN)."""
    a, b = float(a), float(b)
    if b == 0.0:
        if a == 0.0 or math.isnan(a):
            return math.nan
        return math.copysign(math.inf, a) * math.copysign(1.0, b)
    return a / b


def cexp(x):
    """C exp(): overflow gives inf instead of raising."""
    try:
        return math.exp(x)
    except OverflowError:
        return math.inf


def iround(x):
    """fd.h:17 iround(x) = (int) floor(x + 0.5), x + 0.5 in double."""
    return int(math.floor(float(x) + 0.5))


def c_trunc_div(a, b):
    """C integer division (truncates towards zero)."""
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b > 0) else -q


def minimum_m(mat):
    """util.c minimum_m: scan from mat[1][1] keeping strict improvements, so a
    NaN is never chosen unless it is the first element."""
    first = mat.flat[0]
    if np.isnan(first):
        return f32(first)
    rest = mat[~np.isnan(mat)]
    return f32(min(first, rest.min())) if rest.size else f32(first)


def maximum_m(mat):
    first = mat.flat[0]
    if np.isnan(first):
        return f32(first)
    rest = mat[~np.isnan(mat)]
    return f32(max(first, rest.max())) if rest.size else f32(first)


# ---------------------------------------------------------------------------
# tapers (src/taper_grad.c)
# ---------------------------------------------------------------------------
def gauss_value(a, k, tl):
    """exp(-(1.0/2.0) * (a*k/(tl/2.0)) * (a*k/(tl/2.0))) of taper_grad.c:74/79 with
    float a and int k: a*k in float, the rest in double, stored as float."""
    x = cdiv(float(f32(a) * f32(k)), tl / 2.0)
    return f32(cexp((-0.5 * x) * x))


def vertical_window(gradt):
    """taper_grad.c:58-81: window[1..ifw] of the vertical taper (index 0 unused)."""
    g1, g2, g3, g4 = gradt
    tl, tl2, ifw = g2 - g1, g4 - g3, g4 - g1
    win = np.zeros(max(ifw, 0) + 1, np.float32)
    for i in range(1, ifw + 1):
        win[i] = 1.0
        if i <= tl:
            win[i] = gauss_value(3.0, i - tl, tl)
        if i >= ifw - tl2:
            win[i] = gauss_value(3.0, i - (ifw - tl2), tl2)
    return win


def taper_vertical(nx, ny, gradt):
    """taper_grad.c:83-110: coefficients [NY][NX]; row j gets window[1..] for GRADT1 < i < GRADT4."""
    win = vertical_window(gradt)
    g1, g4 = gradt[0], gradt[3]
    row = np.zeros(nx, np.float32)
    h = 1
    for i in range(1, nx + 1):
        if g1 < i < g4:
            row[i - 1] = win[h]
            h += 1
    return np.repeat(row[None, :], ny, axis=0)


def taper_horizontal(nx, ny, dh, gradt, exp_hor):
    """taper_grad.c:172-244: Gaussian ramp on rows GRADT1..GRADT2, then (j DH)^EXP_TAPER_GRAD_HOR."""
    g1, g2 = gradt[0], gradt[1]
    tl, ifw = g2 - g1, g2 - g1 + 1
    win = np.zeros(max(ifw, 0) + 1, np.float32)
    for i in range(1, ifw + 1):
        win[i] = 1.0
        if i <= tl:
            win[i] = gauss_value(3.0, i - tl, tl)
    col = np.zeros(ny, np.float32)
    h = 1
    for j in range(1, ny + 1):
        t = f32(0.0)
        if g1 <= j <= g2:
            t = win[h]
        if j > g2:
            t = f32(math.pow(float(f32(j) * f32(dh)), float(f32(exp_hor))))
        col[j - 1] = t
        if j >= g1:
            h += 1
    return np.repeat(col[:, None], nx, axis=1)


def source_taper_matrix(srtshape, srtradius, dh):
    """taper_grad.c:330-396: the G x G radial taper around one source and its centre ijc.
    Returns (m [G][G] float32 indexed [iy-1][ix-1], ijc)."""
    S, dh = f32(srtradius), f32(dh)
    G = int(math.ceil(cdiv(2.0 * float(S), float(dh))))
    if G < 5:
        G = 5
    m = np.zeros((G, G), np.float32)
    a = f32(1.0)
    maxrad = f32(math.sqrt((2.0 * float(S)) * float(S)))
    for j in range(1, G + 1):
        for i in range(1, G + 1):
            x = f32((float(f32(i)) - float(f32(G)) / 2.0 - 0.5) * float(dh))
            y = f32((float(f32(j)) - float(f32(G)) / 2.0 - 0.5) * float(dh))
            rad = f32(math.sqrt(float(f32(x * x) + f32(y * y))))
            if srtshape == 1:
                m[j - 1, i - 1] = f32(math.erf(float(f32(a * rad) / maxrad)))
            elif srtshape == 2:
                m[j - 1, i - 1] = f32(math.log(float(rad))) if rad > 0 else f32(0.0)
    minm = minimum_m(m.T.copy())   # the scan runs i (x) outer, j inner: same set, same first element
    m = (m - minm).astype(np.float32)
    h = G // 2
    edge = np.array([m[0, h - 1], m[h - 1, 0], m[h - 1, G - 1], m[G - 1, h - 1]], np.float32)
    maxm = maximum_m(edge)
    with np.errstate(divide="ignore", invalid="ignore"):
        m = (m / maxm).astype(np.float32)
    m[m > 1.0] = 1.0
    ijc = int(math.ceil(float(f32(G) / f32(2.0))))
    return m, ijc


def source_cell(x, z, dh):
    """grid cell of a source at (x, z) metres: iround(srcpos / DH) with the division in float."""
    return iround(f32(x) / f32(dh)), iround(f32(z) / f32(dh))


def source_mask(nx, ny, m, ijc, i, j):
    """mm of taper_grad.c:404-420: 1 everywhere, the G x G matrix around (i, j) where it is inside the grid."""
    G = m.shape[0]
    mm = np.ones((ny, nx), np.float32)
    for iy in range(1, G + 1):
        for ix in range(1, G + 1):
            xx, yy = i + ix - ijc, j + iy - ijc
            if 1 <= xx <= nx and 1 <= yy <= ny:
                mm[yy - 1, xx - 1] = m[iy - 1, ix - 1]
    return mm


def normalise_msum(msum):
    """taper_grad.c:458-479: (msum - min) / max over the grid."""
    minm = minimum_m(msum)
    msum = (msum - minm).astype(np.float32)
    maxm = maximum_m(msum)
    with np.errstate(divide="ignore", invalid="ignore"):
        return (msum / maxm).astype(np.float32)


def taper_sources(nx, ny, dh, srcs, srtshape, srtradius):
    """taper_grad.c:330-479: coefficients of the radial taper around every source (minimum over sources)."""
    m, ijc = source_taper_matrix(srtshape, srtradius, dh)
    msum = np.ones((ny, nx), np.float32)
    for x, z in srcs:
        i, j = source_cell(x, z, dh)
        mm = source_mask(nx, ny, m, ijc, i, j)
        upd = msum > mm
        msum[upd] = mm[upd]
    return normalise_msum(msum)


def taper_shot(nx, ny, dh, src, srtshape, srtradius):
    """taper_grad_shot.c: the same taper around one shot's source."""
    return taper_sources(nx, ny, dh, [src], srtshape, srtradius)


def zeroed_cells(nx, ny, points, size, need_row):
    """Cells a loop `waveconvtmp[jj][ii] = 0` over (2 size + 1)^2 boxes around `points` reaches.

    The reference's condition is POS == (i - 1) / NX (C division), i.e. 2 - NX <= i <= NX, and the
    same for j; with need_row it also requires jj > 0.  waveconvtmp is matrix(0, NY+1, 0, NX+1), rows
    of NX + 2 floats in one block, so an index ii <= -2 addresses row jj - 1, column NX + 2 + ii.
    Only cells that land in the interior matter (the array is copied back over 1..NX x 1..NY)."""
    cells = set()
    ncol = nx + 2
    for (i1, j1) in points:
        for i in range(i1 - size, i1 + size + 1):
            for j in range(j1 - size, j1 + size + 1):
                if c_trunc_div(i - 1, nx) != 0 or c_trunc_div(j - 1, ny) != 0:
                    continue
                if need_row and j <= 0:
                    continue
                off = j * ncol + i
                r, c = off // ncol, off % ncol
                if 1 <= r <= ny and 1 <= c <= nx:
                    cells.add((r, c))
    return sorted(cells)


def apply_zero(g, cells):
    g = g.copy()
    for (r, c) in cells:
        g[r - 1, c - 1] = 0.0
    return g


def precond_tapers(g, nx, ny, dh, cfg):
    """precond_PSV.c for one parameter class (cls 0 vp, 1 vs, 2 rho): the enabled tapers in the
    reference's order - vertical, horizontal, sources, file.  cfg keys: taper_vert, taper_hor,
    taper_sources, taper_file, gradt (4), exp_hor, srtshape, srtradius, filtsize, srcs [(x, z) m],
    recs [(i, j)], file (3 arrays [NY][NX]), cls."""
    g = np.asarray(g, np.float32)
    if cfg.get("taper_vert"):
        g = (g * taper_vertical(nx, ny, cfg["gradt"])).astype(np.float32)
        pts = [source_cell(x, z, dh) for x, z in cfg.get("srcs", [])]
        g = apply_zero(g, zeroed_cells(nx, ny, pts, 0, False))
        g = apply_zero(g, zeroed_cells(nx, ny, list(cfg.get("recs", [])), 0, False))
    if cfg.get("taper_hor"):
        g = (g * taper_horizontal(nx, ny, dh, cfg["gradt"], cfg["exp_hor"])).astype(np.float32)
    if cfg.get("taper_sources"):
        g = (g * taper_sources(nx, ny, dh, cfg["srcs"], cfg["srtshape"], cfg["srtradius"])).astype(np.float32)
        pts = [source_cell(x, z, dh) for x, z in cfg["srcs"]]
        g = apply_zero(g, zeroed_cells(nx, ny, pts, cfg["filtsize"], True))
    if cfg.get("taper_file"):
        g = (g * np.asarray(cfg["file"][cfg["cls"]], np.float32)).astype(np.float32)
    return g


def shot_taper_apply(g, nx, ny, dh, src, srtshape, srtradius, filtsize):
    """taper_grad_shot.c on one shot gradient: multiply, then zero the FILTSIZE box."""
    g = (np.asarray(g, np.float32) * taper_shot(nx, ny, dh, src, srtshape, srtradius)).astype(np.float32)
    return apply_zero(g, zeroed_cells(nx, ny, [source_cell(src[0], src[1], dh)], filtsize, True))


# ---------------------------------------------------------------------------
# smooth_grad (src/smooth_grad.c): SPATFILTER 2, 3, 4
# ---------------------------------------------------------------------------
def tripd_factor(d, e):
    """util.c tripd, decomposition part (float): returns the factored (d, e)."""
    d, e = d.astype(np.float32).copy(), e.astype(np.float32).copy()
    for k in range(1, len(d)):
        t = e[k - 1]
        e[k - 1] = f32(t / d[k - 1])
        d[k] = f32(d[k] - f32(t * e[k - 1]))
    return d, e


def tripd_solve(d, e, b):
    """util.c tripd, substitution part, for many right-hand sides b[:, k] at once (float)."""
    b = b.astype(np.float32).copy()
    n = len(d)
    for k in range(1, n):
        b[:, k] = (b[:, k] - (e[k - 1] * b[:, k - 1]).astype(np.float32)).astype(np.float32)
    b[:, n - 1] = (b[:, n - 1] / d[n - 1]).astype(np.float32)
    for k in range(n - 1, 0, -1):
        b[:, k - 1] = ((b[:, k - 1] / d[k - 1]).astype(np.float32) - (e[k - 1] * b[:, k]).astype(np.float32)).astype(np.float32)
    return b


def one_plus(x):
    """`1.0 + x` with float x, stored to float: the sum in double, rounded once."""
    return f32(1.0 + float(x))


def smooth2(g, wd_damp, wd_damp1):
    """smooth2.c:28-166 on the global gradient g [NY][NX]; r1 = WD_DAMP smooths along z,
    r2 = WD_DAMP1 along x.  The reference smooths its work array v[0..NX][0..NY] over the
    index ranges 0..n-1 (index 0 is a zero row/column of the array, the last grid
    row/column is left as it is), which is restated here literally."""
    ny, nx = g.shape
    n1, n2 = ny, nx
    r1 = f32(float(f32(f32(wd_damp) * f32(wd_damp))) * 0.25)
    r2 = f32(float(f32(f32(wd_damp1) * f32(wd_damp1))) * 0.25)
    v = np.zeros((n2 + 1, n1 + 1), np.float32)        # v[ix][iz]
    v[1:, 1:] = np.asarray(g, np.float32).T
    w = f32(1.0)
    # along x, for every iz = 0..n1-1
    d = np.full(n2, one_plus(f32(r2 * f32(w + w))), np.float32)
    e = np.full(n2, f32(-r2 * w), np.float32)
    d[0] = f32(d[0] - f32(r2 * w))
    d[n2 - 1] = one_plus(f32(r2 * w))
    fd, fe = tripd_factor(d, e[: n2 - 1])
    rhs = v[0:n2, 0:n1].T.copy()                       # [iz][ix]
    v[0:n2, 0:n1] = tripd_solve(fd, fe, rhs).T
    # along z, for every ix = 0..n2-1: unknowns iz = 1..n1-1, v[ix][0] a fixed boundary value
    n = n1 - 1
    d = np.full(n, one_plus(f32(r1 * f32(w + w))), np.float32)
    e = np.full(n, f32(-r1 * w), np.float32)
    d[n - 1] = one_plus(f32(r1 * w))
    fd, fe = tripd_factor(d, e[: n - 1])
    rhs = v[0:n2, 1:n1].copy()                         # [ix][iz-1]
    rhs[:, 0] = (rhs[:, 0] + (f32(r1 * w) * v[0:n2, 0]).astype(np.float32)).astype(np.float32)
    v[0:n2, 1:n1] = tripd_solve(fd, fe, rhs)
    return v[1:, 1:].T.copy()


def clamp_shift(g, dj, di):
    """g[clamp(j + dj)][clamp(i + di)]: the edge-replicated extension of gauss_filt.c:93-124."""
    ny, nx = g.shape
    jj = np.clip(np.arange(ny) + dj, 0, ny - 1)
    ii = np.clip(np.arange(nx) + di, 0, nx - 1)
    return g[jj][:, ii]


def gauss_size(wd_damp, vel, fc_end, dh):
    """round((WD_DAMP * (vel / FC_END)) / DH), every operation in float, round() of C."""
    lam = f32(f32(vel) / f32(fc_end))
    q = f32(f32(f32(wd_damp) * lam) / f32(dh))
    return int(math.floor(abs(float(q)) + 0.5)) * (1 if q >= 0 else -1)


def gauss_kernel(hfs_x, hfs_z):
    """kernel weights exp(-(ii*ii)/sx - (jj*jj)/sz) (ii*ii / s in float, exp in double, stored as float)
    for ii in -hfs_x..hfs_x, jj in -hfs_z..hfs_z; sigma = hfs/2 in integer arithmetic."""
    sx = f32(2.0 * float(f32(hfs_x // 2)) * float(f32(hfs_x // 2)))
    sz = f32(2.0 * float(f32(hfs_z // 2)) * float(f32(hfs_z // 2)))
    k = np.zeros((2 * hfs_x + 1, 2 * hfs_z + 1), np.float32)      # [ii][jj]
    with np.errstate(divide="ignore", invalid="ignore"):
        for ii in range(-hfs_x, hfs_x + 1):
            for jj in range(-hfs_z, hfs_z + 1):
                a = f32(f32(ii * ii) / sx)
                b = f32(f32(jj * jj) / sz)
                k[ii + hfs_x, jj + hfs_z] = f32(cexp(float(f32(-a - b))))
    return k


def gauss_filt(g, wd_damp, fc_end, c_vs, dh):
    """gauss_filt.c:52-165 (SPATFILTER 3).  The reference accumulates the kernel sum in a
    variable it never initialises; it is started at 0 here."""
    g = np.asarray(g, np.float32)
    F = gauss_size(wd_damp, c_vs, fc_end, dh)
    if F == 0:
        return g.copy()
    if F % 2 == 0:
        F = F + 1 if F > 0 else F - 1
    hfs = abs(F) // 2
    k = gauss_kernel(hfs, hfs)
    s = f32(0.0)
    for ii in range(2 * hfs + 1):
        for jj in range(2 * hfs + 1):
            s = f32(s + k[ii, jj])
    if F > 0:
        k = (k / s).astype(np.float32)
    conv = np.zeros_like(g)
    for ii in range(-hfs, hfs + 1):
        for jj in range(-hfs, hfs + 1):
            conv = (conv + (clamp_shift(g, jj, ii) * k[ii + hfs, jj + hfs]).astype(np.float32)).astype(np.float32)
    return conv


def gauss_filt_var(g, vel, wd_damp, wd_damp1, fc_end, dh):
    """gauss_filt_var.c:82-190 (SPATFILTER 4): per cell a Gaussian whose x and z sizes follow the
    local wavelength vel / FC_END (vel = the S-velocity model, [NY][NX]).  Cells closer to the edge
    than the z half-size read edge-replicated values (the reference pads by the x half-size of the
    fastest cell only, so for WD_DAMP1 > WD_DAMP it would read outside its padded copy)."""
    g = np.asarray(g, np.float32)
    vel = np.asarray(vel, np.float32)
    ny, nx = g.shape
    out = g.copy()
    sizes = {}
    for j in range(ny):
        for i in range(nx):
            fx = gauss_size(wd_damp, vel[j, i], fc_end, dh)
            fz = gauss_size(wd_damp1, vel[j, i], fc_end, dh)
            if fz <= 0:
                continue
            if fx % 2 == 0:
                fx += 1
            if fz % 2 == 0:
                fz += 1
            fx, fz = max(fx, 6), max(fz, 6)
            sizes.setdefault((abs(fx) // 2, abs(fz) // 2), []).append((j, i))
    for (hx, hz), cells in sizes.items():
        k = gauss_kernel(hx, hz)
        js = np.array([c[0] for c in cells])
        is_ = np.array([c[1] for c in cells])
        conv = np.zeros(len(cells), np.float32)
        s = f32(0.0)
        for ii in range(-hx, hx + 1):
            for jj in range(-hz, hz + 1):
                w = k[ii + hx, jj + hz]
                vals = g[np.clip(js + jj, 0, ny - 1), np.clip(is_ + ii, 0, nx - 1)]
                conv = (conv + (vals * w).astype(np.float32)).astype(np.float32)
                s = f32(s + w)
        out[js, is_] = (conv / s).astype(np.float32)
    return out


def smooth_grad(g, spatfilter, wd_damp, wd_damp1, fc_end, c_vs, dh, vel=None):
    """smooth_grad.c: SPATFILTER 2 smooth2, 3 gauss_filt, 4 gauss_filt_var (1 needs FFTW)."""
    if spatfilter == 2:
        return smooth2(g, wd_damp, wd_damp1)
    if spatfilter == 3:
        return gauss_filt(g, wd_damp, fc_end, c_vs, dh)
    if spatfilter == 4:
        return gauss_filt_var(g, vel, wd_damp, wd_damp1, fc_end, dh)
    return np.asarray(g, np.float32).copy()
