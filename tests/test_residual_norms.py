"""Objective functions of calc_res that need no FFT (LNORM 1, 2, 3, 4, 5, 7, 8
with COMP_WEIGHT, TRKILL, OFFSET_MUTE, N_ORDER, TIMEWIN 5): the oracle
(oracle/residual_oracle.py) against the reference's own calc_res."""
import os
import sys

import numpy as np
import pytest

import oracles as O

sys.path.insert(0, os.path.join(O.ROOT, "oracle"))
import residual_oracle as ro  # noqa: E402

needs_ref = pytest.mark.skipif(not O.reference_available(), reason="reference build not present")

NTR, NS, DT, DH = 12, 300, 1e-3, 5.0


def sections(seed=0):
    rng = np.random.default_rng(seed)
    t = np.arange(NS) * DT
    base = np.sin(2 * np.pi * 15 * t)[None, :] * (1.0 + rng.random((NTR, 1)))
    syn = (base * 1e-3 + 1e-5 * rng.standard_normal((NTR, NS))).astype(np.float32)
    obs = (np.roll(base, 3, axis=1) * 1.2e-3 + 1e-5 * rng.standard_normal((NTR, NS))).astype(np.float32)
    obs[4, 10:20] = syn[4, 10:20]            # equal samples: the L1 sign is 0 there
    return obs, syn


REC = (np.arange(10, 10 + 6 * NTR, 6).astype(np.int32), np.full(NTR, 3, np.int32))
SRC = (150.0, 10.0)

# (lnorm, grad_form, mode, n_order, comp_weight, trkill, offset_mute, timewin)
CASES = [
    (1, 1, 1, 0, 0, 0, 0, 0), (2, 1, 1, 0, 0, 0, 0, 0), (2, 2, 1, 0, 0, 0, 0, 0), (2, 1, 2, 0, 0, 0, 0, 0),
    (2, 2, 2, 0, 0, 0, 0, 0), (2, 1, 1, 2, 1, 1, 1, 0), (2, 2, 3, 1, 0, 0, 2, 5), (3, 1, 1, 0, 0, 0, 0, 0),
    (4, 2, 1, 0, 0, 0, 0, 0), (5, 1, 1, 0, 0, 0, 0, 0), (5, 2, 1, 1, 1, 0, 0, 0), (7, 1, 1, 0, 0, 0, 0, 0),
    (7, 2, 1, 0, 0, 1, 0, 0), (8, 2, 1, 0, 0, 0, 0, 0), (8, 2, 1, 1, 1, 0, 1, 0),
]
FOPT = (3500.0, 2200.0, 120.0, 40.0, 1500.0, 5.0, 25.0)   # c_vp, c_rho, offsetc, gamma, twlength_minus, fc_start, fc_end
KILL = np.array([0, 1, 0, 0, 0, 1, 0, 0, 0, 0, 0, 1], np.int32)


def oracle_call(case, obs, syn):
    ln, gf, mode, no, cw, tk, om, tw = case
    return ro.calc_res(obs, syn, DT, lnorm=ln, grad_form=gf, mode=mode, n_order=no, comp_weight=cw, c_vp=FOPT[0],
                       c_rho=FOPT[1], kill=KILL if tk else None, offset_mute=om, offsetc=FOPT[2], timewin=tw,
                       gamma=FOPT[3], twlength_minus=FOPT[4], fc_start=FOPT[5], fc_end=FOPT[6], rec=REC, src=SRC,
                       dh=DH)


@needs_ref
@pytest.mark.parametrize("case", CASES, ids=[f"L{c[0]}gf{c[1]}m{c[2]}n{c[3]}cw{c[4]}k{c[5]}om{c[6]}tw{c[7]}"
                                            for c in CASES])
def test_oracle_matches_reference(tmp_path, case):
    obs, syn = sections(case[0])
    want, wl2 = O.run_isolated(O.ref_calc_res_ex, str(tmp_path), obs, syn, DT, DH, case, FOPT, REC[0], REC[1], SRC,
                               KILL if case[5] else None)
    got, l2 = oracle_call(case, obs, syn)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    assert l2 == wl2
