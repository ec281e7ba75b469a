"""FWI outer loop on the CPU: step length and model update against the
reference's calc_opt_step / calc_mat_change_test_PSV, and the step-length
search logic of step_length_est_psv."""
import ctypes

import numpy as np
import pytest

import oracles as O
from denise_b200 import fwi

needs_ref = pytest.mark.skipif(not O.reference_available(), reason="reference build not present")


def _ref_opt(L2t, epst):
    lib = ctypes.CDLL(O.REF_SO)
    lib.refh_calc_opt_step.restype = ctypes.c_float
    return lib.refh_calc_opt_step((ctypes.c_double * 3)(*L2t), (ctypes.c_float * 3)(*epst))


def _ref_mat(vp, vs, rho, g, eps_scale, lim, it, inv, scalerho):
    lib = ctypes.CDLL(O.REF_SO)
    nx, ny = vp.shape
    outs = [np.empty_like(vp) for _ in range(3)]
    eps = np.zeros(3, np.float32)
    lim = np.asarray(lim, np.float32)
    inv = np.asarray(inv, np.int32)
    lib.refh_mat_change(nx, ny, *[O._fp(np.ascontiguousarray(a)) for a in (vp, vs, rho, *g)],
                        ctypes.c_float(eps_scale), O._fp(lim), it, O._ip(inv), ctypes.c_float(scalerho),
                        *[O._fp(o) for o in outs], O._fp(eps))
    return outs, eps


CASES = [
    ([1.0, 0.5, 0.8], [0.0, 0.01, 0.02]),      # interior minimum
    ([1.0, 0.7, 0.4], [0.0, 0.01, 0.02]),      # still descending: clamp to the last step
    ([1.0, 1.2, 1.1], [0.0, 0.01, 0.02]),      # maximum
    ([2.0, 1.0, 3.0], [0.0, 0.005, 0.0075]),
]


@needs_ref
@pytest.mark.parametrize("L2t,epst", CASES)
def test_calc_opt_step_matches_reference(L2t, epst):
    ours = fwi.calc_opt_step(L2t, epst)
    ref = O.run_isolated(_ref_opt, L2t, epst)
    # the reference solves the 3x3 system in float, this build in double
    assert abs(ours - ref) <= 1e-4 * max(abs(ref), 1e-6), (ours, ref)


@needs_ref
@pytest.mark.parametrize("it,inv", [(1, (1, 1, 1)), (2, (1, 3, 1))])
def test_mat_update_matches_reference(it, inv):
    rng = np.random.default_rng(it)
    nx, ny = 40, 30
    vp = rng.uniform(1500, 4500, (nx, ny)).astype(np.float32)
    vs = (vp / 1.8).astype(np.float32)
    vs[:, :3] = 0.0                                   # water: vs below the lower limit but <= 1e-6
    rho = rng.uniform(1800, 2600, (nx, ny)).astype(np.float32)
    g = [rng.standard_normal((nx, ny)).astype(np.float32) * s for s in (1e-3, 2e-3, 5e-4)]
    lim = (1400.0, 4600.0, 600.0, 2600.0, 1700.0, 2700.0)
    ours = fwi.mat_update(vp, vs, rho, *g, 0.02, lim, it, inv, 1.5)
    ref, reps = O.run_isolated(_ref_mat, vp, vs, rho, g, 0.02, lim, it, inv, 1.5)
    for a, b in zip(ours[:3], ref):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(np.asarray(ours[3], np.float32), reps)


def test_step_length_brackets_a_parabola():
    f = lambda e: (e - 0.013) ** 2 + 0.1
    eps, L2t, epst, found = fwi.step_length(f, f(0.0), 0.01, 2.0, 4)
    assert found and abs(eps - 0.013) < 1e-6
    assert L2t[1] < L2t[0]


def test_step_length_shrinks_when_the_first_test_is_worse():
    f = lambda e: (e - 0.002) ** 2
    eps, L2t, epst, found = fwi.step_length(f, f(0.0), 0.01, 2.0, 4)
    assert found and abs(eps - 0.002) < 1e-6 and epst[1] < 0.01


def test_step_length_gives_up():
    eps, L2t, epst, found = fwi.step_length(lambda e: 1.0 + e, 1.0, 0.01, 2.0, 3)
    assert not found
