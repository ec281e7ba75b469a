"""FWI outer loop on the GPU: the FP64 L-BFGS direction against a numpy
restatement of the two-loop recursion, the secant condition, the deterministic
dot product, and two FWI iterations lowering the misfit of a small problem."""
import numpy as np
import pytest

from denise_b200 import fwi, synth

import oracles as O
from test_gpu_serve import _request

pytestmark = pytest.mark.gpu


def _two_loop(S, Y, g):
    """Nocedal & Wright algorithm 7.4 with H0 = (s.y / y.y) I of the newest pair."""
    q = g.copy()
    rho = [1.0 / (y @ s) if (y @ s) != 0 else 0.0 for s, y in zip(S, Y)]
    alpha = [0.0] * len(S)
    for k in reversed(range(len(S))):
        alpha[k] = rho[k] * (S[k] @ q)
        q -= alpha[k] * Y[k]
    r = (S[-1] @ Y[-1]) / (Y[-1] @ Y[-1]) * q
    for k in range(len(S)):
        beta = rho[k] * (Y[k] @ r)
        r += S[k] * (alpha[k] - beta)
    return r


def test_lbfgs_direction_and_secant():
    import torch

    rng = np.random.default_rng(0)
    n, m = 50_000, 5
    A = rng.uniform(0.5, 4.0, n)                  # a diagonal SPD Hessian
    L = fwi.LBFGS(n, m, 0)
    xs = [rng.standard_normal(n) for _ in range(m + 3)]
    S, Y = [], []
    for a, b in zip(xs[:-1], xs[1:]):
        s, y = b - a, A * (b - a)
        L.push(s, y)
        S.append(s)
        Y.append(y)
    S, Y = S[-m:], Y[-m:]
    assert L.count() == m
    g = A * xs[-1]
    r = L.direction(g)
    want = _two_loop(S, Y, g)
    assert np.linalg.norm(r - want) <= 1e-10 * np.linalg.norm(want)
    # secant: H y_newest = s_newest
    assert np.linalg.norm(L.direction(Y[-1]) - S[-1]) <= 1e-9 * np.linalg.norm(S[-1])
    L.close()
    a = torch.as_tensor(rng.standard_normal(1_000_003)).cuda()
    b = torch.as_tensor(rng.standard_normal(1_000_003)).cuda()
    d1, d2 = fwi.dot(a, b), fwi.dot(a, b)
    assert d1 == d2
    assert abs(d1 - float(a.cpu().numpy() @ b.cpu().numpy())) <= 1e-10 * abs(d1)


def test_two_fwi_iterations_lower_the_misfit():
    import denise_b200 as dn

    req = _request(0, "gradient", 90, 60, 500, 8, 0, 4, 11)
    p = req.params
    vp, vs, rho = req.model
    vpt, vst, rhot = synth.add_ellipse(vp, vs, rho, p.dh, 3, v=3600.0)
    # observed data from the true model
    m = dn.Model(p.replace(store_snapshots=0), vpt, vst, rhot)
    ss = [dn.Shot(m, *sh[:5]) for sh in req.shots]
    dn.run(ss)
    obs = [(s.sections(dn.SEC_VX), s.sections(dn.SEC_VY)) for s in ss]
    for s in ss:
        s.close()
    m.close()
    start = tuple(synth.smoothed(a, 3.0) for a in (vp, vs, rho))
    lim = (1000.0, 6000.0, 500.0, 3500.0, 1000.0, 3500.0)
    f = fwi.FWI(p, start, req.shots, obs, lim, device=0, nlbfgs=5, eps_scale=0.01)
    L0 = f.iterate(1)
    L1 = f.iterate(2)
    L2 = f.misfit((f.vp, f.vs, f.rho))
    assert all(h["found"] for h in f.history), f.history
    assert L1 < L0 and L2 < L1, (L0, L1, L2)
    f.close()


def test_fwi_with_gradient_conditioning():
    """The same two iterations with the reference's usual conditioning on: a
    horizontal taper below the sources, smooth2 and the per-shot circular taper;
    the conditioned gradient is the plan applied to the stacked one."""
    import denise_b200 as dn
    from denise_b200.precond import PrecondConfig, PrecondPlan
    from denise_b200.shard import sharded_gradient

    req = _request(0, "gradient", 90, 60, 500, 8, 0, 4, 11)
    p = req.params
    vp, vs, rho = req.model
    vpt, vst, rhot = synth.add_ellipse(vp, vs, rho, p.dh, 3, v=3600.0)
    m = dn.Model(p.replace(store_snapshots=0), vpt, vst, rhot)
    ss = [dn.Shot(m, *sh[:5]) for sh in req.shots]
    dn.run(ss)
    obs = [(s.sections(dn.SEC_VX), s.sections(dn.SEC_VY)) for s in ss]
    for s in ss:
        s.close()
    m.close()
    start = tuple(synth.smoothed(a, 3.0) for a in (vp, vs, rho))
    lim = (1000.0, 6000.0, 500.0, 3500.0, 1000.0, 3500.0)
    cfg = PrecondConfig(spatfilter=2, wd_damp=1.0, wd_damp1=1.0, taper_hor=1, gradt=(5, 9, 0, 0),
                        exp_taper_grad_hor=1.0)
    taper = (1, 4.0 * p.dh, 1)
    f = fwi.FWI(p, start, req.shots, obs, lim, device=0, nlbfgs=5, eps_scale=0.01, precond=cfg, shot_taper=taper)
    g = f.gradient()
    raw = sharded_gradient(p, start, req.shots, obs, None, 0, taper)
    dm = dn.Model(p.replace(store_snapshots=0), *start)
    dm.set_gradient(*[x.astype(np.float32) for x in raw[:3]])
    plan = PrecondPlan(p.nx, p.ny, p.dh, cfg)
    plan.apply(dm)
    for a, b in zip(g[:3], dm.gradient()):
        np.testing.assert_array_equal(a.astype(np.float32), b)
    assert np.abs(g[0][:, :4]).max() == 0.0          # the taper zeroes rows above GRADT1
    dm.close()
    plan.close()
    L0 = f.iterate(1)
    L1 = f.iterate(2)
    assert all(h["found"] for h in f.history), f.history
    assert L1 < L0, (L0, L1)
    f.close()


def test_fwi_with_time_filter():
    """TIME_FILT: sources and observed data are band-limited before the iteration."""
    import denise_b200 as dn

    req = _request(0, "gradient", 90, 60, 500, 8, 0, 4, 11)
    p = req.params
    vp, vs, rho = req.model
    vpt, vst, rhot = synth.add_ellipse(vp, vs, rho, p.dh, 3, v=3600.0)
    m = dn.Model(p.replace(store_snapshots=0), vpt, vst, rhot)
    ss = [dn.Shot(m, *sh[:5]) for sh in req.shots]
    dn.run(ss)
    obs = [(s.sections(dn.SEC_VX), s.sections(dn.SEC_VY)) for s in ss]
    for s in ss:
        s.close()
    m.close()
    start = tuple(synth.smoothed(a, 3.0) for a in (vp, vs, rho))
    lim = (1000.0, 6000.0, 500.0, 3500.0, 1000.0, 3500.0)
    f = fwi.FWI(p, start, req.shots, obs, lim, device=0, nlbfgs=5, eps_scale=0.01, time_filter=(4, 30.0, 2.0))
    np.testing.assert_array_equal(f.shots[0][2], dn.tdfilt(req.shots[0][2], p.dt, 4, 30.0, 2.0))
    np.testing.assert_array_equal(f.obs[1][0], dn.tdfilt(obs[1][0], p.dt, 4, 30.0, 2.0))
    L0 = f.iterate(1)
    assert np.isfinite(L0) and f.history[0]["found"]
    f.close()


def test_workflow_two_stages(tmp_path):
    """A two-stage workflow file: a 25 Hz low-pass L2 stage with smooth2, then a
    full-band stage with the energy preconditioning and the global-correlation
    misfit; each stage runs up to two iterations and lowers its misfit."""
    import denise_b200 as dn
    from denise_b200 import workflow

    req = _request(0, "gradient", 90, 60, 500, 8, 0, 4, 11)
    p = req.params
    vp, vs, rho = req.model
    vpt, vst, rhot = synth.add_ellipse(vp, vs, rho, p.dh, 3, v=3600.0)
    m = dn.Model(p.replace(store_snapshots=0), vpt, vst, rhot)
    ss = [dn.Shot(m, *sh[:5]) for sh in req.shots]
    dn.run(ss)
    obs = [(s.sections(dn.SEC_VX), s.sections(dn.SEC_VY)) for s in ss]
    for s in ss:
        s.close()
    m.close()
    start = tuple(synth.smoothed(a, 3.0) for a in (vp, vs, rho))
    lim = (1000.0, 6000.0, 500.0, 3500.0, 1000.0, 3500.0)
    wf = tmp_path / "workflow.inp"
    wf.write_text(" ".join(workflow.STAGE_KEYS) + "\n"
                  "0.001 1 0.0 25.0 4 0 0.0 0.0 0.0 1 1 1 0 2 1.0 1.0 0 2 0 0 0.0 0.0 0 0 0.0 1.0 1.0 0 0.0 0\n"
                  "0.001 0 0.0 40.0 4 0 0.0 0.0 0.0 1 1 1 0 0 0.0 0.0 1 5 0 0 0.0 0.0 0 0 0.0 1.0 1.0 0 0.0 0\n")
    stages = workflow.read_workflow(str(wf))
    assert len(stages) == 2
    prefix, log = str(tmp_path / "model"), str(tmp_path / "misfit.dat")
    vp1, vs1, rho1, res = workflow.run_workflow(p, start, req.shots, obs, lim, stages, itermax=2, nlbfgs=5,
                                                out_prefix=prefix, misfit_log=log)
    assert [r.stage for r in res] == [1, 2]
    for r in res:
        assert r.iterations >= 1 and all(np.isfinite(r.misfits))
        if len(r.misfits) == 2 and r.reason == "ITERMAX":
            assert r.misfits[1] < r.misfits[0] or r.misfits[1] <= 0.0, r
    assert not np.array_equal(vp1, start[0])
    # model files per stage (x-major float32) and one log line per iteration with the stage number
    stage2 = [np.fromfile(x, np.float32).reshape(p.nx, p.ny) for x in workflow.stage_files(prefix, 2)]
    np.testing.assert_array_equal(stage2[0], vp1)
    np.testing.assert_array_equal(stage2[2], rho1)
    lines = open(log).read().splitlines()
    assert len(lines) == sum(r.iterations for r in res)
    assert [int(x.split()[-1]) for x in lines] == [r.stage for r in res for _ in range(r.iterations)]
    # a second run resumes after stage 2 from its files: nothing left to do
    vp2, vs2, rho2, res2 = workflow.run_workflow(p, start, req.shots, obs, lim, stages, itermax=2, nlbfgs=5,
                                                 out_prefix=prefix, resume=True)
    assert [r.reason for r in res2] == ["resumed", "resumed"]
    np.testing.assert_array_equal(vp2, vp1)
