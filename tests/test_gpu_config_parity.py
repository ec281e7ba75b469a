"""Parity at the benchmark workloads' full sizes, not only on small grids:

* C0, the plain elastic forward (600 x 300, NT 5000, FDORDER 8, free
  surface, 120 receivers): the GPU sections against the reference's own code,
  bit for bit;
* C1, one shot of the batched viscoelastic workload (2000 x 600, L = 3, 600
  steps): the same;
* C2, the FWI gradient (1700 x 500, NT 4000, DTINV 2) of two of its 32 shots
  against observed data of the true model: the GPU FP32 gradient against the
  reference's grad_obj_psv shot loop (forward, calc_res, adjoint, ass_gradPSV,
  stacked in shot order) bit for bit, and the GPU gradient with FP16 snapshots
  against the FP64 restatement (double wavefields and snapshots, the same
  adjoint sources) within 1e-3 relative L2, the north-star bar.

The reference runs are long CPU jobs (minutes at C2 size); they start in
spawned processes when the module starts and run while the GPU works.  The C2
reference shots keep 34 GB of snapshots each and the FP64 oracle 68 GB per
shot in host memory, so those tests skip on a host without that memory free."""
import multiprocessing as mp
import os
import sys
from concurrent.futures import ProcessPoolExecutor

import numpy as np
import pytest

import config_cases as CC
import oracles as O
import denise_b200 as dn
from denise_b200 import synth

sys.path.insert(0, os.path.join(O.ROOT, "oracle"))
import residual_oracle as ro  # noqa: E402

pytestmark = [pytest.mark.gpu, pytest.mark.slow,
              pytest.mark.skipif(not O.reference_available(), reason="reference build not present")]

C1_NT = 600
C2_PICK = (0, 16)          # two of the 32 shot positions


def _gpu_sections(p, model, src, rec):
    m = dn.Model(p, *model[:3], model[3] if p.L else None, model[4] if p.L else None)
    s = dn.Shot(m, *src[:3], *rec)
    dn.run([s])
    out = s.sections(dn.SEC_VX), s.sections(dn.SEC_VY)
    s.close()
    m.close()
    return out


@pytest.fixture(scope="module")
def jobs():
    """Reference jobs in spawned processes, started before the GPU runs of the module."""
    ex = ProcessPoolExecutor(max_workers=4, mp_context=mp.get_context("spawn"))
    futs = {}
    p0, model0, src0, rec0 = synth.c0_case(seed=0)
    futs["c0"] = ex.submit(CC.ref_forward, p0, model0, src0, rec0)
    p1 = synth.c1_params(nt=C1_NT)
    model1, src1, rec1 = synth.c1_shot(p1, 5)
    futs["c1"] = ex.submit(CC.ref_forward, p1, model1, src1, rec1)
    # C2: observed data of the two shots from the true model, on the GPU, then the reference's gradients
    p2, true, start, shots = CC.c2_case()
    picked = [shots[k] for k in C2_PICK]
    obs = []
    mt = dn.Model(p2.replace(store_snapshots=0), *true)
    for sh in picked:
        s = dn.Shot(mt, *sh)
        dn.run([s])
        obs.append((s.sections(dn.SEC_VX), s.sections(dn.SEC_VY)))
        s.close()
    mt.close()
    need = len(picked) * CC.snapshot_bytes(p2, 4)
    c2 = dict(p=p2, start=start, shots=picked, obs=obs)
    if CC.available_memory() > 1.3 * need:
        c2["ref"] = [ex.submit(CC.ref_gradient_shot, p2, start, sh, ob[0], ob[1]) for sh, ob in zip(picked, obs)]
    cases = dict(c0=(p0, model0, src0, rec0), c1=(p1, model1, src1, rec1), c2=c2)
    yield ex, futs, cases
    ex.shutdown(wait=True, cancel_futures=True)


def test_c0_full_size_matches_reference(jobs):
    _, futs, cases = jobs
    vx, vy = _gpu_sections(*cases["c0"])
    rvx, rvy, secs = futs["c0"].result(timeout=1800)
    np.testing.assert_array_equal(vx, rvx)
    np.testing.assert_array_equal(vy, rvy)
    assert np.abs(vy).max() > 0


def test_c1_shot_matches_reference(jobs):
    _, futs, cases = jobs
    vx, vy = _gpu_sections(*cases["c1"])
    rvx, rvy, secs = futs["c1"].result(timeout=1800)
    np.testing.assert_array_equal(vx, rvx)
    np.testing.assert_array_equal(vy, rvy)
    assert np.abs(vy).max() > 0


def _gpu_gradient(p, start, shots, obs, prec):
    """Stacked GPU gradient of the shots with the L2 adjoint sources computed from
    this run's sections (calc_res, restated in oracle/residual_oracle.py, which the
    device residual equals bit for bit)."""
    m = dn.Model(p.replace(snap_precision=prec), *start)
    ss = [dn.Shot(m, *sh) for sh in shots]
    dn.run(ss, dn.MODE_FORWARD)
    res = []
    for s, (ovx, ovy) in zip(ss, obs):
        rvx, _ = ro.calc_res(ovx, s.sections(dn.SEC_VX), p.dt)
        rvy, _ = ro.calc_res(ovy, s.sections(dn.SEC_VY), p.dt)
        s.set_residuals(rvx, rvy, None)
        res.append((rvx, rvy))
    dn.run(ss, dn.MODE_ADJOINT)
    for s in ss:
        s.accumulate_gradient()
        s.close()
    g = m.gradient()
    m.close()
    return g, res


def test_c2_gradient_matches_reference(jobs):
    _, futs, cases = jobs
    c2 = cases["c2"]
    if "ref" not in c2:
        pytest.skip("host memory below the reference's snapshot arrays")
    ours, _ = _gpu_gradient(c2["p"], c2["start"], c2["shots"], c2["obs"], dn.SNAP_F32)
    stacked = [np.zeros_like(ours[0]) for _ in range(3)]
    for f in c2["ref"]:
        g = f.result(timeout=3600)
        for a, b in zip(stacked, g[:3]):
            a += b                     # waveconv += waveconv_shot in float, in shot order (grad_obj_psv.c:253-261)
    for a, b, name in zip(ours, stacked, ("vp", "vs", "rho")):
        np.testing.assert_array_equal(a, b, err_msg=name)
        assert np.abs(b).max() > 0


def test_c2_fp16_gradient_vs_fp64_oracle(jobs):
    ex, futs, cases = jobs
    c2 = cases["c2"]
    for f in c2.get("ref", []):       # the reference shots first: their snapshots leave host memory
        f.result(timeout=3600)
    if CC.available_memory() < 1.3 * CC.snapshot_bytes(c2["p"], 8):
        pytest.skip("host memory below the FP64 oracle's snapshot arrays")
    g16, res = _gpu_gradient(c2["p"], c2["start"], c2["shots"], c2["obs"], dn.SNAP_F16)
    ref = ex.submit(CC.fp64_gradient, c2["p"], c2["start"], c2["shots"], res).result(timeout=3600)
    errs = [O.rel_l2(a, b) for a, b in zip(g16, ref[:3])]
    assert max(errs) < 1e-3, errs
