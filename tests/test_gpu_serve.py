"""Continuous batching: requests of different sizes, physics and modes run
through the serving loop, with later requests joining queues that are already
running; every result must be identical (bit for bit) to the same request run
alone through the batch API."""
import numpy as np
import pytest

import denise_b200 as dn
from denise_b200 import serve, synth

pytestmark = pytest.mark.gpu


def _request(rid, kind, nx, ny, nt, fdorder, L, nshots, seed):
    p = synth.c0_params(nx=nx, ny=ny, nt=nt, fw=10, L=L, fl=(2.0, 8.0, 25.0)[:L], ts=0.1, fdorder=fdorder,
                        store_snapshots=1 if kind == "gradient" else 0, dtinv=2)
    vp, vs, rho = synth.base_model(nx, ny, p.dh, seed)
    model = (vp, vs, rho) + (synth.q_model(nx, ny, seed) if L else ())
    sig = synth.ricker_source(p, 40.0)[None, :] * 1e3
    nr = (nx - 10) // 6
    rec = (np.arange(5, 5 + 6 * nr, 6).astype(np.int32), np.full(nr, 4, np.int32))
    shots = [(np.array([nx // 3 + 7 * k], np.int32), np.array([3], np.int32), sig) + rec for k in range(nshots)]
    obs = None
    if kind == "gradient":
        rng = np.random.default_rng(seed)
        obs = [tuple((1e-9 * rng.standard_normal((nr, nt))).astype(np.float32) for _ in range(2))
               for _ in range(nshots)]
    return serve.Request(kind, p, model, shots, obs, rid=rid)


def _alone(req):
    p = req.params
    m = dn.Model(p, *req.model[:3], req.model[3] if p.L else None, req.model[4] if p.L else None)
    shots = [dn.Shot(m, *sh[:5]) for sh in req.shots]
    if req.kind == "forward":
        dn.run(shots, dn.MODE_FORWARD)
        out = [{"vx": s.sections(dn.SEC_VX), "vy": s.sections(dn.SEC_VY)} for s in shots]
    else:
        misfits = []
        for s, (ovx, ovy) in zip(shots, req.obs):
            dn.run([s], dn.MODE_FORWARD)
            misfits.append(s.residual(ovx, dn.SEC_VX) + s.residual(ovy, dn.SEC_VY))
            dn.run([s], dn.MODE_ADJOINT)
        for s in shots:
            s.accumulate_gradient()
        out = (m.gradient(), float(sum(misfits)))
    for s in shots:
        s.close()
    m.close()
    return out


def test_results_are_the_same_alone_and_in_the_mix():
    reqs = [
        _request(0, "forward", 96, 64, 300, 8, 0, 2, 1),
        _request(1, "forward", 80, 60, 250, 4, 2, 1, 2),
        _request(2, "gradient", 72, 56, 280, 8, 0, 2, 3),
        _request(3, "forward", 128, 40, 400, 8, 0, 1, 4),
        _request(4, "gradient", 64, 48, 220, 4, 2, 1, 5),
        _request(5, "forward", 70, 70, 260, 12, 0, 1, 6),
    ]
    srv = serve.Server(device=0, chunk=20)
    for r in reqs[:3]:
        srv.submit(r)
    srv.step()
    srv.step()
    for r in reqs[3:]:
        srv.submit(r)
    results = {r.rid: r for r in srv.run()}
    st = srv.stats()
    srv.close()
    assert len(results) == len(reqs)
    assert st["joins_while_running"] >= 1 and st["max_running_shots"] >= 2, st
    for req in reqs:
        res = results[req.rid]
        assert res.status == 0
        alone = _alone(req)
        if req.kind == "forward":
            for a, b in zip(res.sections, alone):
                np.testing.assert_array_equal(a["vx"], b["vx"])
                np.testing.assert_array_equal(a["vy"], b["vy"])
        else:
            for a, b in zip(res.gradient, alone[0]):
                np.testing.assert_array_equal(a, b)
            assert res.misfit == alone[1]
    assert st["p99_s"] >= st["p50_s"] > 0
