"""The reference's FWI optimisers on the CPU: the numpy restatement
(oracle/optim_oracle.py) against the reference's own store_LBFGS_PSV / LBFGS /
extract_LBFGS_PSV and descent / store_PCG_PSV / PCG / extract_PCG_PSV
(FWI_PSV.c:637-676, called through oracle/ref_harness.c), iteration after
iteration with a pointer wrap and a stage reset, bit for bit with float dot
products.  With the FP64 dot products of the device the directions stay within
1e-4 relative L2 of the reference's (its float sums over 3 nx ny products carry
relative errors of order 1e-5)."""
import ctypes
import os
import sys

import numpy as np
import pytest

import oracles as O

sys.path.insert(0, os.path.join(O.ROOT, "oracle"))
from optim_oracle import ReferenceOptimizer  # noqa: E402

needs_ref = pytest.mark.skipif(not O.reference_available(), reason="reference build not present")

NX, NY = 23, 17


def _iterates(n, seed):
    """A sequence of models drifting and gradients varying smoothly, as an inversion's."""
    rng = np.random.default_rng(seed)
    base = [rng.uniform(lo, hi, (NX, NY)).astype(np.float32) for lo, hi in ((2000, 4000), (1200, 2300), (1900, 2600))]
    g0 = [rng.standard_normal((NX, NY)).astype(np.float32) * s for s in (1e-3, 2e-3, 5e-4)]
    out = []
    for k in range(n):
        model = [(b * (1 + 0.01 * k) + rng.standard_normal((NX, NY)) * 3).astype(np.float32) for b in base]
        grads = [(g * (0.8 ** k) + rng.standard_normal((NX, NY)) * 1e-4 * s).astype(np.float32)
                 for g, s in zip(g0, (1, 2, 0.5))]
        out.append((model, grads))
    return out


def _reference_run(workdir, method, nlbfgs, pcg_beta, its, c, reset_after):
    os.chdir(workdir)
    lib = ctypes.CDLL(O.REF_SO)
    lib.refh_optim_init(method, NX, NY, nlbfgs, pcg_beta, b"jac")
    out, it = [], 0
    for k, (model, grads) in enumerate(its):
        it += 1
        g = [np.ascontiguousarray(x).copy() for x in grads]
        lib.refh_optim_step(it, O._fp(np.asarray(c, np.float32)), *[O._fp(np.ascontiguousarray(m)) for m in model],
                            *[O._fp(x) for x in g])
        files = {}
        if method == 2:
            for name in ("p", "p_u", "p_rho", "p_vp", "p_vs", "p_mrho", "c", "c_u", "c_rho"):
                files[name] = np.fromfile(f"jac_{name}.old", np.float32).reshape(NX, NY)
                assert np.array_equal(files[name], np.fromfile(f"jac_{name}.old.0.0", np.float32).reshape(NX, NY))
        out.append((g, files))
        if k + 1 == reset_after:
            lib.refh_optim_reset()
            it = 0
    return out


def _oracle_run(method, nlbfgs, pcg_beta, its, c, reset_after, dots):
    o = ReferenceOptimizer(method, NX, NY, nlbfgs, pcg_beta, dots)
    out, it = [], 0
    for k, (model, grads) in enumerate(its):
        it += 1
        d = o.step(it, c, model, grads)
        out.append((d, {n: v.reshape(NX, NY) for n, v in o.files.items()}))
        if k + 1 == reset_after:
            o.reset()
            it = 0
    return out


CASES = [(2, 3, 2, 7, 5), (2, 20, 2, 4, 0), (1, 0, 1, 4, 0), (1, 0, 2, 5, 3), (1, 0, 3, 4, 0), (1, 0, 4, 4, 0)]


@needs_ref
@pytest.mark.parametrize("method,nlbfgs,pcg_beta,n,reset_after", CASES)
def test_optimizer_restatement_matches_reference(tmp_path, method, nlbfgs, pcg_beta, n, reset_after):
    its = _iterates(n, 7 + method + pcg_beta)
    c = (3001.25, 1733.5, 2240.75)
    ref = O.run_isolated(_reference_run, str(tmp_path), method, nlbfgs, pcg_beta, its, c, reset_after)
    ours = _oracle_run(method, nlbfgs, pcg_beta, its, c, reset_after, "float")
    fp64 = _oracle_run(method, nlbfgs, pcg_beta, its, c, reset_after, "fp64")
    for k, ((rd, rf), (od, of), (fd, _)) in enumerate(zip(ref, ours, fp64)):
        for a, b in zip(rd, od):
            assert np.array_equal(a, b), f"iteration {k + 1}: direction differs"
        for name, v in rf.items():
            assert np.array_equal(v, of[name]), f"iteration {k + 1}: JACOBIAN_{name}.old differs"
        for a, b in zip(rd, fd):
            assert O.rel_l2(b, a) < 1e-4, f"iteration {k + 1}: FP64 dots moved the direction"
