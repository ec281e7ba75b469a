"""Gradient conditioning on the GPU (dn_precond_apply, the per-shot circular
taper of dn_shot_accumulate_gradient_ex) against the oracle restatement of
smooth_grad / precond_PSV / taper_grad_shot, which tests/test_precond.py pins
to the reference's own functions: float gradients must come out bit for bit."""
import os
import sys

import numpy as np
import pytest

import denise_b200 as dn
from denise_b200 import synth
from denise_b200.precond import PrecondConfig, PrecondPlan

import oracles as O
from test_gpu_parity import _residuals, gpu_shot, small_case

sys.path.insert(0, os.path.join(O.ROOT, "oracle"))
import precond_oracle as po  # noqa: E402

pytestmark = pytest.mark.gpu

NX, NY, DH = 96, 64, 5.0
SRCS = [(0.0, 40.0), (150.0, 30.0), (477.0, 5.0), (3.0, 60.0), (240.0, 200.0)]
RECS = [(5, 4), (20, 4), (96, 10), (1, 1), (50, 64)]
GRADT = (3, 9, 80, 90)


def bits_equal(a, b):
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    same = (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))
    return int((~same).sum())


def model_with_gradient(seed, grad_accum=dn.ACC_F32, nx=NX, ny=NY):
    p = synth.c0_params(nx=nx, ny=ny, nt=10, fw=10, grad_accum=grad_accum)
    vp, vs, rho = synth.base_model(nx, ny, DH, seed)
    m = dn.Model(p, vp, vs, rho)
    rng = np.random.default_rng(seed)
    g = [rng.standard_normal((nx, ny)).astype(np.float32) for _ in range(3)]   # file order
    m.set_gradient(*g)
    return m, g, vs


CONFIGS = {
    "tapers": dict(taper_vert=1, taper_hor=1, taper_sources=1, srtshape=1, srtradius=12.0, filtsize=3),
    "tapers_log": dict(taper_sources=1, srtshape=2, srtradius=22.0, filtsize=1),
    "smooth2": dict(spatfilter=2, wd_damp=2.0, wd_damp1=3.0, taper_hor=1),
    "gauss": dict(spatfilter=3, wd_damp=1.0, fc_end=10.0, c_vs=400.0, taper_vert=1),
    "gauss_var": dict(spatfilter=4, wd_damp=0.4, wd_damp1=0.3, fc_end=25.0, taper_sources=1, srtshape=1,
                      srtradius=8.0, filtsize=2),
    "file": dict(taper_file=1),
}


def oracle(g_file, vs_file, c: PrecondConfig, files):
    """oracle result for one class (file-order input, [NY][NX] output)"""
    out = []
    for cls, g in enumerate(g_file):
        x = po.smooth_grad(g.T, c.spatfilter, c.wd_damp, c.wd_damp1, c.fc_end, c.c_vs, DH, vs_file.T)
        cfg = dict(taper_vert=c.taper_vert, taper_hor=c.taper_hor, taper_sources=c.taper_sources,
                   taper_file=c.taper_file, gradt=c.gradt, exp_hor=c.exp_taper_grad_hor, srtshape=c.srtshape,
                   srtradius=c.srtradius, filtsize=c.filtsize, srcs=c.sources, recs=c.receivers,
                   file=[f.T for f in files] if files else None, cls=cls)
        out.append(po.precond_tapers(x, NX, NY, DH, cfg))
    return out


@pytest.mark.parametrize("name", list(CONFIGS))
def test_conditioning_bitexact(name):
    m, g, vs = model_with_gradient(3)
    rng = np.random.default_rng(11)
    files = [rng.random((NX, NY)).astype(np.float32) for _ in range(3)] if name == "file" else None
    c = PrecondConfig(gradt=GRADT, exp_taper_grad_hor=1.5, sources=SRCS, receivers=RECS, taper_files=files,
                      **CONFIGS[name])
    plan = PrecondPlan(NX, NY, DH, c)
    plan.apply(m)
    got = m.gradient()
    want = oracle(g, vs, c, files)
    for cls in range(3):
        assert bits_equal(got[cls].T, want[cls]) == 0, (name, cls)
    plan.apply(m)          # applying twice conditions twice (the plan is reusable)
    again = m.gradient()
    want2 = oracle([w.T for w in want], vs, c, files)
    for cls in range(3):
        assert bits_equal(again[cls].T, want2[cls]) == 0, (name, cls)
    plan.close()
    m.close()


def test_conditioning_double_gradient_close():
    m, g, vs = model_with_gradient(4, grad_accum=dn.ACC_F64)
    c = PrecondConfig(gradt=GRADT, exp_taper_grad_hor=1.5, sources=SRCS, receivers=RECS, **CONFIGS["gauss_var"])
    plan = PrecondPlan(NX, NY, DH, c)
    plan.apply(m)
    got = m.gradient()
    want = oracle(g, vs, c, None)
    for cls in range(3):
        assert O.rel_l2(got[cls].T, want[cls]) < 1e-6
    plan.close()
    m.close()


def test_conditioning_large_grid_properties():
    """8000 x 500: smoothing keeps a constant field constant away from the
    reference's untouched last row/column; tapers of 1 leave it unchanged."""
    nx, ny = 8000, 500
    p = synth.c0_params(nx=nx, ny=ny, nt=10, fw=10)
    vp, vs, rho = synth.base_model(nx, ny, DH, 1)
    m = dn.Model(p, vp, vs, rho)
    one = np.ones((nx, ny), np.float32)
    m.set_gradient(one, one, one)
    plan = PrecondPlan(nx, ny, DH, PrecondConfig(spatfilter=3, wd_damp=1.0, fc_end=10.0, c_vs=400.0))
    plan.apply(m)
    got = m.gradient()[0]
    assert np.abs(got - 1.0).max() < 1e-5
    plan.close()
    m.close()


def test_shot_circular_taper_bitexact():
    p, model, src, rec = small_case(store_snapshots=1)
    ref = O.Restatement(p, model, src, rec, "f")
    ref.forward(store=True)
    rvx, rvy = _residuals(p, ref.sections(0), ref.sections(1))
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    s.set_residuals(rvx, rvy, None)
    dn.run([s], dn.MODE_ADJOINT)
    s.accumulate_gradient()
    plain = m.gradient()
    m.zero_gradient()
    sx, sz = float(src[0][0]) * p.dh, float(src[1][0]) * p.dh
    s.accumulate_gradient_ex(circular_taper=(1, 3.0 * p.dh, 2, sx, sz))
    got = m.gradient()
    for a, b in zip(got, plain):
        want = po.shot_taper_apply(b.T, p.nx, p.ny, p.dh, (sx, sz), 1, 3.0 * p.dh, 2)
        want = (np.float32(0.0) + want).astype(np.float32)      # stacked onto a zero gradient
        assert bits_equal(a.T, want) == 0
    m.close()
