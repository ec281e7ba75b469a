"""ORACLE / TEST INFRASTRUCTURE - never part of the product.

Restatement of the reference's time-domain filter apply_tdfilt
(src/apply_tdfilt.c:10-20) -> timedomain_filt (src/timedomain_filt.c) ->
seife_lpb / seife_hpb of the libcseife library vendored in the reference tree
(libcseife/cseife.c:41-51, :139-177; libcseife/cseife_rfk.c; libcseife/
cseife_rekfl.c).  The published algorithm is E. Wielandt's recursive
Butterworth filter of seife (bilinear transform): an order-m filter is one
first-order section (m odd) followed by m/2 second-order sections with damping
h_j = sin(pi/2 (2j - 1) / m), each applied as
    y_k = f0 x_k + f1 x_{k-1} + f2 x_{k-2} + g1 y_{k-1} + g2 y_{k-2}
from rest, with eps = 2 pi / (T0 / dt) and
    first order:  g1 = (2 - eps) / (2 + eps); low-pass f0 = f1 = eps / (2 + eps);
                  high-pass f0 = 2 / (2 + eps), f1 = -f0
    second order: a = 1 - eps h + eps^2/4, b = -2 + eps^2/2, c = 1 + eps h + eps^2/4,
                  g1 = -b / c, g2 = -a / c; low-pass f0 = eps^2/4/c, f1 = 2 f0, f2 = f0;
                  high-pass f0 = 1/c, f1 = -f0 - f0, f2 = f0.
timedomain_filt copies a trace into a double vector allocated from index 1
and hands the filter the pointer of index 0 (a zero), so the filter runs over
[0, d_1, ..., d_{ns-1}] and the last sample d_ns passes unfiltered; the high
pass subtracts that leading zero (seife_first), which changes nothing.
Everything in double with the C library's atan and sin; pinned against the
reference's apply_tdfilt in tests/test_tdfilt.py.
"""
import math

import numpy as np


def sections(order, t0_samples, highpass):
    """[(f0, f1, f2, g1, g2)] of seife_butterworth for period t0 (in samples)."""
    one, two, four, eight = 1.0, 2.0, 4.0, 8.0
    zpi = eight * math.atan(one)
    eps = zpi / t0_samples
    out = []
    mm = order // 2
    if order > 2 * mm:
        g1 = (two - eps) / (two + eps)
        if highpass:
            f0 = two / (two + eps)
            out.append((f0, -f0, 0.0, g1, 0.0))
        else:
            f0 = eps / (two + eps)
            out.append((f0, f0, 0.0, g1, 0.0))
    pih = 2.0 * math.atan(1.0)
    for j in range(1, mm + 1):
        h = math.sin(pih * (2 * j - 1) / order)
        epsq = eps * eps
        a = one - eps * h + epsq / four
        b = -two + epsq / two
        c = one + eps * h + epsq / four
        g1, g2 = -b / c, -a / c
        if highpass:
            f0 = one / c
            out.append((f0, -f0 - f0, f0, g1, g2))
        else:
            f0 = epsq / four / c
            out.append((f0, f0 + f0, f0, g1, g2))
    return out


def recurse(x, coef):
    """seife_rekfl on a list of doubles, in place semantics (returns a new list)."""
    f0, f1, f2, g1, g2 = coef
    xa = xaa = ya = yaa = 0.0
    y = []
    for xn in x:
        v = f0 * xn + f1 * xa + f2 * xaa + g1 * ya + g2 * yaa
        xaa, xa, yaa, ya = xa, xn, ya, v
        y.append(v)
    return y


def timedomain_filt(data, fc, order, dt, method):
    """timedomain_filt.c on [ntr][ns] float32 data; method 1 low-pass, 2 high-pass."""
    data = np.asarray(data, np.float32)
    out = data.copy()
    t0 = 1.0 / float(np.float32(fc))
    secs = sections(order, t0 / float(np.float32(dt)), method == 2)
    for i in range(data.shape[0]):
        x = [0.0] + [float(v) for v in data[i, :-1]]      # the leading zero, without the last sample
        if method == 2:
            x0 = x[0]
            x = [v - x0 for v in x]
        for c in secs:
            x = recurse(x, c)
        out[i, :-1] = np.array(x[1:], np.float64).astype(np.float32)
    return out


def apply_tdfilt(data, dt, order, fc2, fc1):
    """apply_tdfilt.c: low-pass at fc2, then high-pass at fc1 if fc1 > 0."""
    out = timedomain_filt(data, fc2, order, dt, 1)
    if fc1 > 0.0:
        out = timedomain_filt(out, fc1, order, dt, 2)
    return out
