"""The reference's optimisers on the device (dn_optim_*) against their numpy
restatement with the same FP64 dot products (oracle/optim_oracle.py, pinned to
the reference's store_LBFGS_PSV / LBFGS / extract_LBFGS_PSV and PCG in
tests/test_optim.py): the search direction and the JACOBIAN vectors of every
iteration, through pointer wraps and stage resets, for L-BFGS and all four
PCG_BETA rules, with float and double gradient accumulators.  The two sum the
exact double products in different orders, so a dot product may round to a
neighbouring float: the directions agree to 1e-6 relative L2."""
import os
import sys

import numpy as np
import pytest

import oracles as O
from denise_b200 import api as dn
from denise_b200 import fwi, synth

sys.path.insert(0, os.path.join(O.ROOT, "oracle"))
from optim_oracle import ReferenceOptimizer  # noqa: E402

pytestmark = pytest.mark.gpu

NX, NY = 61, 37


def _iterates(n, seed):
    rng = np.random.default_rng(seed)
    vp, vs, rho = synth.base_model(NX, NY, 5.0, seed)
    g0 = [rng.standard_normal((NX, NY)).astype(np.float32) * s for s in (1e-3, 2e-3, 5e-4)]
    out = []
    for k in range(n):
        model = [(a * (1 + 0.004 * k) + rng.standard_normal((NX, NY)) * 2).astype(np.float32) for a in (vp, vs, rho)]
        grads = [(g * (0.8 ** k) + rng.standard_normal((NX, NY)) * 1e-4 * s).astype(np.float32)
                 for g, s in zip(g0, (1, 2, 0.5))]
        out.append((model, grads))
    return out


@pytest.mark.parametrize("method,nlbfgs,pcg_beta,n,reset_after,acc",
                         [(2, 3, 2, 7, 5, 0), (2, 20, 2, 4, 0, 1), (1, 0, 1, 4, 0, 0), (1, 0, 2, 5, 3, 0),
                          (1, 0, 3, 4, 0, 1), (1, 0, 4, 4, 0, 0)])
def test_device_optimizer_matches_restatement(method, nlbfgs, pcg_beta, n, reset_after, acc):
    p = synth.c0_params(nx=NX, ny=NY, nt=10, fw=5, grad_accum=acc)
    c = (3001.25, 1733.5, 2240.75)
    dev = fwi.Optimizer(method, NX, NY, nlbfgs, pcg_beta, 0)
    ref = ReferenceOptimizer(method, NX, NY, nlbfgs, pcg_beta, "fp64")
    it = 0
    for k, (model, grads) in enumerate(_iterates(n, 3 + method + pcg_beta)):
        it += 1
        m = dn.Model(p, *model, device=0)
        m.set_gradient(*grads)
        dev.step(m, it, c)
        got = m.gradient()
        want = ref.step(it, c, model, grads)
        for a, b in zip(got, want):
            assert O.rel_l2(a, b) < 1e-6, (k, O.rel_l2(a, b))
        if method == 2:
            for w, name in enumerate(fwi.Optimizer.FILES):
                assert O.rel_l2(dev.vector(w), ref.files[name].reshape(NX, NY)) < 1e-6, (k, name)
            assert np.array_equal(dev.vector(3), model[0]) and np.array_equal(dev.vector(5), model[2])
        m.close()
        if k + 1 == reset_after:
            dev.reset()
            ref.reset()
            it = 0
    dev.close()


def test_first_lbfgs_step_is_the_normalised_gradient():
    """Iteration 1 (and the first after a reset) of L-BFGS: the direction is C g
    bit for bit (store_LBFGS_PSV.c:37-85 without the L-BFGS update)."""
    p = synth.c0_params(nx=NX, ny=NY, nt=10, fw=5)
    (model, grads), = _iterates(1, 9)
    c = (2900.0, 1650.5, 2210.25)
    o = fwi.Optimizer(2, NX, NY, 5, 2, 0)
    m = dn.Model(p, *model, device=0)
    m.set_gradient(*grads)
    o.step(m, 1, c)
    for g, d, cc in zip(grads, m.gradient(), c):
        assert np.array_equal(d, (np.float32(cc) * g).astype(np.float32))
    m.close()
    o.close()
