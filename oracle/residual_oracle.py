"""ORACLE / TEST INFRASTRUCTURE - never part of the product.

numpy/Python restatement of the reference's data residual and misfit,
calc_res() (src/calc_res.c:7-640), for the objective functions that need no
Fourier transform: LNORM 1 (L1 sign, :423-430), 2 (L2, :432-453), 3 (Cauchy,
:455-458), 4 (sech, :460-462), 5 (global correlation, :130-157, :331-360,
:465-490), 7 (normalised integration, :240-303, :362-382) and 8 (AGC-weighted
L2 for GRAD_FORM 2, :47-55, :386-398, :505-513), with COMP_WEIGHT (:92-127),
TRKILL (:58-84), OFFSET_MUTE (:306-323), N_ORDER (:400-414) and TIMEWIN 5
(:440-443).

Float operations are spelled out in float32, double ones in Python floats,
with sqrt/tanh/exp/pow from the C library via math; the misfit is one double
accumulated over traces and samples in the reference's order.  Sections are
[ntr][ns] float32; the residual comes back time-reversed as calc_res leaves it.
Pinned against the reference's own calc_res (tests/test_residual_norms.py).
"""
import math

import numpy as np

f32 = np.float32


def _iround(x):
    return int(math.floor(float(x) + 0.5))


def calc_res(data, syn, dt, lnorm=2, grad_form=1, mode=1, n_order=0, comp_weight=0, c_vp=0.0, c_rho=0.0,
             kill=None, offset_mute=0, offsetc=0.0, timewin=0, gamma=0.0, twlength_minus=1.0, fc_start=0.0,
             fc_end=0.0, rec=None, src=(0.0, 0.0), dh=1.0):
    """Returns (residual [ntr][ns] float32, misfit float)."""
    d_all = np.array(data, np.float32, copy=True)
    s_all = np.array(syn, np.float32, copy=True)
    ntr, ns = d_all.shape
    dt = f32(dt)
    res = np.zeros((ntr, ns), np.float32)
    L2 = 0.0
    if comp_weight > 0:
        w = f32(f32(c_vp) * f32(c_rho))
        s_all = (s_all * w).astype(np.float32)
        d_all = (d_all * w).astype(np.float32)

    def integrate(a):
        out = np.zeros_like(a)
        acc = f32(0.0)
        for j in range(len(a)):
            acc = f32(acc + a[j])
            out[j] = f32(dt * acc)
        return out

    integ = lnorm == 5 and grad_form == 1 or lnorm == 7
    if integ:
        if grad_form == 1:
            is_s = [integrate(s_all[i]) for i in range(ntr)]
            is_d = [integrate(d_all[i]) for i in range(ntr)]
        else:
            is_s = [s_all[i].copy() for i in range(ntr)]
            is_d = [d_all[i].copy() for i in range(ntr)]
    if lnorm == 7:
        qm, qt, dq = [], [], []
        for i in range(ntr):
            a, b = np.zeros(ns, np.float32), np.zeros(ns, np.float32)
            Qm = Qt = f32(0.0)
            for j in range(ns):
                Qm = f32(Qm + f32(is_s[i][j] * is_s[i][j]))
                Qt = f32(Qt + f32(is_d[i][j] * is_d[i][j]))
                a[j], b[j] = Qm, Qt
            with np.errstate(divide="ignore", invalid="ignore"):
                a = (a / Qm).astype(np.float32)
                b = (b / Qt).astype(np.float32)
            qm.append(a)
            qt.append(b)
            dq.append((a - b).astype(np.float32))
    nagc = 0
    if lnorm == 8 and grad_form == 2:
        nagc = _iround(2.0 / float(f32(f32(f32(fc_start) + f32(fc_end)) * dt)))
    agc = np.zeros((ntr, ns), np.float32)
    offsets = np.zeros(ntr, np.float32)
    for i in range(ntr):
        if kill is not None and kill[i] == 1:
            continue
        s, d = s_all[i], d_all[i]
        if offset_mute or timewin == 5:
            xr = f32(f32(rec[0][i]) * f32(dh))
            yr = f32(f32(rec[1][i]) * f32(dh))
            xs, ys = f32(src[0]), f32(src[1])
            dx, dy = f32(xs - xr), f32(ys - yr)
            off = f32(math.sqrt(float(f32(f32(dx * dx) + f32(dy * dy)))))
            offsets[i] = off
            if offset_mute == 1 and off >= f32(offsetc):
                continue
            if offset_mute == 2 and off <= f32(offsetc):
                continue
        if lnorm == 5:
            ad = asn = dms = f32(0.0)
            for j in range(ns):
                xd = d[j] if grad_form == 2 else is_d[i][j]
                xs_ = s[j] if grad_form == 2 else is_s[i][j]
                ad = f32(ad + f32(xd * xd))
                asn = f32(asn + f32(xs_ * xs_))
                dms = f32(dms + f32(xs_ * xd))
            ad = f32(math.sqrt(float(ad)))
            asn = f32(math.sqrt(float(asn)))
        if lnorm == 7:
            Q1 = Q2 = f32(0.0)
            for j in range(ns):
                Q1 = f32(Q1 + f32(dq[i][j] * qm[i][j]))
                Q2 = f32(Q2 + qm[i][j])
            Q3 = f32(0.0)
            h = 0
            for j in range(ns - 1, -1, -1):
                Q3 = f32(Q3 + dq[i][j])
                res[i, h] = f32((-2.0 * float(is_s[i][j])) * float(f32(f32(-Q3) - Q1)) / float(Q2))
                h += 1
        if lnorm == 8 and grad_form == 2:
            for j in range(ns):
                a = f32(0.0)
                for hh in range(j - nagc, j + nagc + 1):
                    if 0 <= hh < ns:
                        a = f32(a + f32(d[hh] * d[hh]))
                agc[i, j] = f32(math.sqrt(float(a)))
        for _ in range(n_order):
            d[0] = f32(d[0] * dt)
            s[0] = f32(s[0] * dt)
            for j in range(1, ns):
                d[j] = f32(d[j - 1] + f32(d[j] * dt))
                s[j] = f32(s[j - 1] + f32(s[j] * dt))
        intseis = f32(0.0)
        sign = f32(0.0)
        for j in range(ns):
            inv = ns - 1 - j
            if j == 0:
                d[0] = s[0]
            if lnorm == 1:
                df = f32(d[j] - s[j])
                if df > 0:
                    sign = f32(1.0)
                if df < 0:
                    sign = f32(-1.0)
                if df == 0:
                    sign = f32(0.0)
                res[i, inv] = sign
            if lnorm == 2:
                if grad_form == 1:
                    intseis = f32(intseis + f32(dt * (f32(s[j] - d[j]) if mode != 2 else d[j])))
                else:
                    intseis = f32(s[j] - d[j]) if mode != 2 else d[j]
                res[i, inv] = intseis
                if timewin == 5:
                    t0 = f32(abs(float(f32(offsets[i] / f32(twlength_minus)))))
                    tj = f32(f32(j + 1) * dt)
                    if tj >= t0:
                        e = math.exp(-float(f32(gamma)) * math.pow(float(f32(tj - t0)), 2))
                        res[i, inv] = f32(float(res[i, inv]) * e)
            if lnorm == 3:
                df = f32(d[j] - s[j])
                res[i, inv] = f32(df / f32(f32(1.0) + f32(df * df)))
            if lnorm == 4:
                res[i, inv] = f32(math.tanh(float(f32(d[j] - s[j]))))
            if lnorm == 5:
                xd = d[j] if grad_form == 2 else is_d[i][j]
                xs_ = s[j] if grad_form == 2 else is_s[i][j]
                tmp = f32(f32(f32(asn * asn) * asn) * ad)
                tmp1 = f32(asn * ad)
                with np.errstate(divide="ignore", invalid="ignore"):
                    res[i, inv] = f32(f32(f32(xs_ * dms) / f32(tmp + f32(0.0))) - f32(xd / f32(tmp1 + f32(0.0))))
                    L2 -= float(f32(f32(xd * xs_) / f32(f32(ad * asn) + f32(0.0))))
            if lnorm == 8 and grad_form == 2:
                v = f32(0.0)
                if abs(agc[i, j]) > 0.0:
                    v = f32(f32(s[j] - d[j]) / agc[i, j])
                res[i, inv] = v
        # the misfit loop of calc_res.c:521-600 (same traces)
        for j in range(ns):
            inv = ns - 1 - j
            if lnorm == 2:
                L2 += 0.5 * float(res[i, inv]) * float(res[i, inv])
            if lnorm == 7:
                L2 += 0.5 * float(dq[i][inv]) * float(dq[i][inv])
            if lnorm == 8 and grad_form == 2 and abs(agc[i, j]) > 0.0:
                df = float(f32(s[j] - d[j]))
                L2 += 0.5 * df * df / float(agc[i, j])
    return res, L2
