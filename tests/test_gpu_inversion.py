"""MODE 1 of a parameter file with a workflow file, end to end: the reference's
own program (oracle/_ref/denise, CPU) and ``python -m denise_b200`` (GPU) run
the same one-stage FWI from a smoothed starting model against data of the true
model, with the per-shot circular gradient taper, for four iterations with
L-BFGS (GRAD_METHOD 2) and with PCG (GRAD_METHOD 1).  Compared: every line of
the misfit log (opteps, the three test steps, L2t[1..4], the stage), the
models after every iteration (INV_MOD_OUT 1) and after the last update
(INV_MODELFILE_*.bin), and the L-BFGS JACOBIAN files.  Iteration 1 is the same
arithmetic on both sides except the grouping of the misfit's double sums; from
iteration 2 on, the optimisers' dot products are summed in FP64 here and in
float by the reference (relative differences of order 1e-5 in the direction),
so the comparisons carry tolerances.  LOG = 1: with LOG = 0 the reference's
FWI writes to a log handle that has been closed and aborts ("invalid stdio
handle").  A case without the shot taper is not used: there the reference's
own gradient points uphill for every step it tries (its step search fails in
iteration 1)."""
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

import oracles as O
import inp_case
from denise_b200 import io, synth, workflow

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NX, NY, DH = 100, 64, 5.0
ITERS = 4
STAGE = "0.01 0 0.0 0.0 4 0 0.0 0.0 0.0 0 0 0 0 0 0.0 0.0 0 2 0 0 0.0 0.0 0 0 0.0 1.0 1.0 0 0.0 0\n"
FWI = dict(MODE=1, NX=NX, NY=NY, DH=DH, TIME=0.12, ITERMAX=ITERS, DATA_DIR="su/obs", TESTSHOT=[1, 2, 1],
           INV_MOD_OUT=1, INV_MODELFILE="model/inv", MISFIT_LOG_FILE="L2_LOG.dat", SEIS_FILE_VX="su/fwi_x.su",
           SEIS_FILE_VY="su/fwi_y.su", VPUPPERLIM=6000.0, VPLOWERLIM=1000.0, VSUPPERLIM=4000.0, VSLOWERLIM=0.0,
           RHOUPPERLIM=3500.0, RHOLOWERLIM=1000.0, GRAD_METHOD=2, PCG_BETA=2, NLBFGS=5, EPS_SCALE=0.01,
           STEPMAX=4, SCALEFAC=2.0, MIN_ITER=2, DTINV=2, TFILE="taper/taper", LOG=1, JACOBIAN="jacobian/gradient",
           SWS_TAPER_CIRCULAR_PER_SHOT=1, SRTSHAPE=1, SRTRADIUS=25.0, FILTSIZE=2)


def _make(root, grad_method):
    """True-model data through the forward driver (bit-identical to the reference's
    program, tests/test_gpu_driver.py), then the smoothed starting model and the
    FWI parameter and workflow files."""
    inp_case.write_case(root, nx=NX, ny=NY, dh=DH, nshots=2, nrec=24, TIME=0.12, SEIS_FILE_VX="su/obs_x.su",
                        SEIS_FILE_VY="su/obs_y.su")
    cwd = os.getcwd()
    try:
        os.chdir(root)
        io.forward_inp("case.inp", 0)
    finally:
        os.chdir(cwd)
    for ext in ("vp", "vs", "rho"):
        path = os.path.join(root, "model", f"test.{ext}")
        a = np.fromfile(path, np.float32).reshape(NX, NY)
        synth.smoothed(a, 4.0).astype(np.float32).tofile(path)
    os.makedirs(os.path.join(root, "taper"), exist_ok=True)
    inp_case.write_inp(os.path.join(root, "case.inp"), **dict(FWI, GRAD_METHOD=grad_method))
    with open(os.path.join(root, "workflow.inp"), "w") as f:
        f.write(" ".join(workflow.STAGE_KEYS) + "\n" + STAGE)


def _log(path):
    return [[float(x) for x in ln.split()] for ln in open(path).read().splitlines() if ln.strip()]


def _bin(root, name):
    return np.fromfile(os.path.join(root, name), np.float32)


@pytest.mark.skipif(not os.path.exists(O.REF_BIN), reason="reference program not built")
@pytest.mark.parametrize("grad_method", [2, 1])
def test_fwi_parameter_file_matches_reference_program(tmp_path, grad_method):
    ref_dir, our_dir = str(tmp_path / "ref"), str(tmp_path / "ours")
    os.makedirs(ref_dir)
    _make(ref_dir, grad_method)
    shutil.copytree(ref_dir, our_dir)
    r = subprocess.run([O.REF_BIN, "case.inp", "workflow.inp"], cwd=ref_dir, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    env = dict(os.environ, PYTHONPATH=os.path.join(ROOT, "denise-black-edition_b200"))
    r = subprocess.run([sys.executable, "-m", "denise_b200", "case.inp", "workflow.inp"], cwd=our_dir,
                       capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    ref_log, our_log = _log(os.path.join(ref_dir, "L2_LOG.dat")), _log(os.path.join(our_dir, "L2_LOG.dat"))
    assert len(ref_log) == len(our_log) == ITERS, (ref_log, our_log)
    for k, (a, b) in enumerate(zip(our_log, ref_log)):
        assert len(a) == len(b) == 9, (a, b)
        # opteps, epst1[1..3]: the same bracketing steps and a parabola minimum close to the reference's
        assert a[1:4] == b[1:4], (k, a, b)
        np.testing.assert_allclose(a[0], b[0], rtol=1e-3 if k else 1e-5, err_msg=f"iteration {k + 1}")
        # L2t[1..4]: the misfits of the current and the test models
        np.testing.assert_allclose(a[4:8], b[4:8], rtol=1e-4 if k else 1e-6, err_msg=f"iteration {k + 1}")
        assert a[8] == b[8] == 1
    assert our_log[-1][7] < 0.5 * our_log[0][7]     # the inversion lowers the misfit
    for it in range(1, ITERS + 1):
        for name in ("vp", "vs", "rho"):
            f = f"model/inv_{name}_stage_1_it_{it}.bin"
            assert O.rel_l2(_bin(our_dir, f), _bin(ref_dir, f)) < 1e-5, f
    for name in ("vp", "vs", "rho"):
        for f in (f"model/inv_{name}.bin", f"model/inv_{name}.bin.0.0"):
            assert O.rel_l2(_bin(our_dir, f), _bin(ref_dir, f)) < 1e-5, f
    if grad_method == 2:
        for name in ("p", "p_u", "p_rho", "p_vp", "p_vs", "p_mrho", "c", "c_u", "c_rho"):
            for suffix in (".old", ".old.0.0"):
                f = f"jacobian/gradient_{name}{suffix}"
                tol = 1e-5 if name in ("p_vp", "p_vs", "p_mrho") else 1e-3
                assert O.rel_l2(_bin(our_dir, f), _bin(ref_dir, f)) < tol, (f, O.rel_l2(_bin(our_dir, f),
                                                                                      _bin(ref_dir, f)))
