"""Device L2 residual / misfit (calc_res, LNORM 2) against the reference.

The adjoint source must be bit-identical to the reference's calc_res() (it is
pure float arithmetic); the misfit is an FP64 sum whose per-trace grouping
differs from the reference's single running sum, so it is compared to 1e-12.
"""
import numpy as np
import pytest

import denise_b200 as dn

import oracles as O
from test_gpu_parity import gpu_shot, small_case

pytestmark = pytest.mark.gpu


def calc_res_numpy(p, data, syn):
    """Float32 restatement of calc_res.c:419-445 (GRAD_FORM 1) and :568."""
    d = data.astype(np.float32).copy()
    d[:, 0] = syn[:, 0]
    res = np.zeros_like(syn, dtype=np.float32)
    acc = np.zeros(syn.shape[0], np.float32)
    l2 = 0.0
    terms = np.zeros_like(res, dtype=np.float64)
    for t in range(p.nt):
        acc = (acc + np.float32(p.dt) * (syn[:, t] - d[:, t]).astype(np.float32)).astype(np.float32)
        res[:, p.nt - 1 - t] = acc
        terms[:, t] = 0.5 * acc.astype(np.float64) * acc.astype(np.float64)
    for r in range(syn.shape[0]):
        for t in range(p.nt):
            l2 += terms[r, t]
    return res, l2


def _ref_calc_res(p, model, src, rec, data, syn):
    r = O.Reference(p, model, src, rec, mode_global=1)
    return r.calc_res(data, syn)


@pytest.mark.parametrize("L", [0, 3])
def test_shot_residual_matches_calc_res(L):
    p, model, src, rec = small_case(L=L, store_snapshots=1)
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    syn = s.sections(dn.SEC_VX)
    rng = np.random.default_rng(5)
    obs = (0.6 * syn + 1e-3 * rng.standard_normal(syn.shape) * np.abs(syn).max()).astype(np.float32)
    l2 = s.residual(obs, dn.SEC_VX)
    res_np, l2_np = calc_res_numpy(p, obs, syn)
    # the shot's adjoint source is internal; run the adjoint with it and compare against the oracle fed
    # with the numpy residual (bit-identical accumulators prove the residuals were identical)
    assert abs(l2 - l2_np) <= 1e-12 * abs(l2_np)
    if O.reference_available():
        res_ref, l2_ref = O.run_isolated(_ref_calc_res, p, model, src, rec, obs, syn)
        np.testing.assert_array_equal(res_np, res_ref)
        assert abs(l2 - l2_ref) <= 1e-12 * abs(l2_ref)
    l2y = s.residual(0.5 * s.sections(dn.SEC_VY), dn.SEC_VY)
    res_y, _ = calc_res_numpy(p, 0.5 * s.sections(dn.SEC_VY), s.sections(dn.SEC_VY))
    assert l2y > 0
    dn.run([s], dn.MODE_ADJOINT)
    ref = O.Restatement(p, model, src, rec, "f")
    ref.forward(store=True)
    ref.adjoint(res_np, res_y, None)
    for fid in (7, 8, 9):
        np.testing.assert_array_equal(s.field(fid), ref.field(fid), err_msg=f"accumulator {fid}")


def test_residual_device_pointers():
    """dn_residual_l2 on raw device buffers (time-major synthetic, trace-major observed)."""
    import ctypes

    import torch

    ntr, nt, dt = 37, 500, 1e-3
    rng = np.random.default_rng(1)
    syn = rng.standard_normal((ntr, nt)).astype(np.float32)
    obs = rng.standard_normal((ntr, nt)).astype(np.float32)
    p = type("P", (), {"nt": nt, "dt": dt})
    res_np, l2_np = calc_res_numpy(p, obs, syn)
    d_syn = torch.from_numpy(np.ascontiguousarray(syn.T)).cuda()
    d_obs = torch.from_numpy(obs).cuda()
    d_res = torch.zeros((ntr, nt), dtype=torch.float32, device="cuda")
    l2 = ctypes.c_double(0.0)
    torch.cuda.synchronize()
    dn._lib.check(dn._lib.lib.dn_residual_l2(d_syn.data_ptr(), d_obs.data_ptr(), d_res.data_ptr(), ntr, nt,
                                             ctypes.c_float(dt), 1, ctypes.byref(l2)))
    np.testing.assert_array_equal(d_res.cpu().numpy(), res_np)
    assert abs(l2.value - l2_np) <= 1e-12 * l2_np


def _ref_rtm_source(p, model, src, rec, data, syn):
    r = O.Reference(p, model, src, rec, mode_global=2)
    return r.calc_res(data, syn)


def test_rtm_source_matches_calc_res_mode2():
    """RTM (MODE 2): the adjoint source is the observed data itself (first sample the
    synthetic one), time-integrated and reversed; bit-identical to the reference."""
    p, model, src, rec = small_case(L=0, store_snapshots=1)
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    syn = s.sections(dn.SEC_VX)
    obs = (0.8 * syn[:, ::-1]).astype(np.float32)
    s.rtm_source(obs, dn.SEC_VX)
    s.rtm_source(0.5 * s.sections(dn.SEC_VY), dn.SEC_VY)
    d = obs.copy()
    d[:, 0] = syn[:, 0]
    want = np.zeros_like(d)
    acc = np.zeros(d.shape[0], np.float32)
    for t in range(p.nt):
        acc = (acc + np.float32(p.dt) * d[:, t]).astype(np.float32)
        want[:, p.nt - 1 - t] = acc
    if O.reference_available():
        ref, _ = O.run_isolated(_ref_rtm_source, p, model, src, rec, obs, syn)
        np.testing.assert_array_equal(want, ref)
    dy = (0.5 * s.sections(dn.SEC_VY)).astype(np.float32)
    dy[:, 0] = s.sections(dn.SEC_VY)[:, 0]
    want_y = np.zeros_like(dy)
    acc = np.zeros(dy.shape[0], np.float32)
    for t in range(p.nt):
        acc = (acc + np.float32(p.dt) * dy[:, t]).astype(np.float32)
        want_y[:, p.nt - 1 - t] = acc
    dn.run([s], dn.MODE_ADJOINT)
    ref = O.Restatement(p, model, src, rec, "f")
    ref.forward(store=True)
    ref.adjoint(want, want_y, None)
    for fid in (7, 8, 9):
        np.testing.assert_array_equal(s.field(fid), ref.field(fid), err_msg=f"accumulator {fid}")
