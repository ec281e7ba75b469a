"""MODE 1 of a parameter file with a workflow file, end to end: the reference's
own program (oracle/_ref/denise, CPU) and ``python -m denise_b200`` (GPU) run
the same one-stage FWI from a smoothed starting model against data of the true
model.  The whole input path (parameter and workflow files, sources, receivers,
wavelets, SU data, test shots, residuals) must give the same misfit of the
starting model.  The search directions differ by design (L-BFGS in FP64 on a
per-class scaled model vector here, the reference's own gradient
normalisation), so the step search is not compared; on this case the
reference's first step fails (opteps 0) while ours finds one.  LOG = 1: with
LOG = 0 the reference's FWI writes to a log handle that has been closed and
aborts ("invalid stdio handle")."""
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
STAGE = "0.01 0 0.0 0.0 4 0 0.0 0.0 0.0 0 0 0 0 0 0.0 0.0 0 2 0 0 0.0 0.0 0 0 0.0 1.0 1.0 0 0.0 0\n"
FWI = dict(MODE=1, NX=NX, NY=NY, DH=DH, TIME=0.12, ITERMAX=1, DATA_DIR="su/obs", TESTSHOT=[1, 2, 1],
           INV_MOD_OUT=1, INV_MODELFILE="model/inv", MISFIT_LOG_FILE="L2_LOG.dat", SEIS_FILE_VX="su/fwi_x.su",
           SEIS_FILE_VY="su/fwi_y.su", VPUPPERLIM=6000.0, VPLOWERLIM=1000.0, VSUPPERLIM=4000.0, VSLOWERLIM=0.0,
           RHOUPPERLIM=3500.0, RHOLOWERLIM=1000.0, GRAD_METHOD=2, NLBFGS=5, EPS_SCALE=0.01, STEPMAX=4,
           SCALEFAC=2.0, MIN_ITER=0, DTINV=2, TFILE="taper/taper", LOG=1)


def _make(root):
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
    inp_case.write_inp(os.path.join(root, "case.inp"), **FWI)
    with open(os.path.join(root, "workflow.inp"), "w") as f:
        f.write(" ".join(workflow.STAGE_KEYS) + "\n" + STAGE)


def _log(path):
    return [[float(x) for x in ln.split()] for ln in open(path).read().splitlines() if ln.strip()]


@pytest.mark.skipif(not os.path.exists(O.REF_BIN), reason="reference program not built")
def test_fwi_parameter_file_matches_reference_program(tmp_path):
    ref_dir, our_dir = str(tmp_path / "ref"), str(tmp_path / "ours")
    os.makedirs(ref_dir)
    _make(ref_dir)
    shutil.copytree(ref_dir, our_dir)
    r = subprocess.run([O.REF_BIN, "case.inp", "workflow.inp"], cwd=ref_dir, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    env = dict(os.environ, PYTHONPATH=os.path.join(ROOT, "denise-black-edition_b200"))
    r = subprocess.run([sys.executable, "-m", "denise_b200", "case.inp", "workflow.inp"], cwd=our_dir,
                       capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    ref_log, our_log = _log(os.path.join(ref_dir, "L2_LOG.dat")), _log(os.path.join(our_dir, "L2_LOG.dat"))
    assert len(ref_log) == len(our_log) == 1 and len(our_log[0]) == len(ref_log[0]) == 9, (ref_log, our_log)
    # opteps, epst1[1..3], L2t[1..4], stage: the misfit of the starting model (L2t[1] = L2t[4])
    np.testing.assert_allclose(our_log[0][4], ref_log[0][4], rtol=1e-5)
    np.testing.assert_allclose(our_log[0][7], ref_log[0][7], rtol=1e-5)
    assert our_log[0][8] == ref_log[0][8] == 1
    if our_log[0][0] > 0:   # a step was found: the model after iteration 1 is written and lowers the misfit
        assert min(our_log[0][5], our_log[0][6] or np.inf) < our_log[0][4]
        for name in ("vp", "vs", "rho"):
            f = os.path.join(our_dir, "model", f"inv_{name}_stage_1_it_1.bin")
            assert os.path.getsize(f) == 4 * NX * NY, f
