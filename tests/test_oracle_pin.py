"""Pins the CPU restatement (oracle/psv_oracle.c) to the reference.

* against the golden fixtures of tests/golden/ (outputs of the reference's own
  compiled code, made by tests/golden/make_golden.py): bit-identical;
* against the live reference build when it is present here;
* the FP64 restatement against the float one: the FP32 rounding error of the
  scheme, stated per quantity.
"""
import numpy as np
import pytest

import oracles as O
from golden.make_golden import CASES, load


@pytest.mark.parametrize("name", sorted(CASES))
def test_float_restatement_matches_reference_golden(name):
    p, model, src, rec, z = load(name)
    r = O.Restatement(p, model, src, rec, "f")
    np.testing.assert_array_equal(r.setup(0), z["hc"])
    np.testing.assert_array_equal(r.setup(1), z["pml"])
    np.testing.assert_array_equal(r.setup(2), z["rip"])
    np.testing.assert_array_equal(r.setup(3), z["rjp"])
    np.testing.assert_array_equal(r.setup(4), z["uipjp"])
    r.forward(store=True)
    for c in range(5):
        np.testing.assert_array_equal(r.sections(c), z[f"sec{c}"], err_msg=f"section {c}")
    for f in range(7):
        np.testing.assert_array_equal(r.field(f), z[f"field{f}"], err_msg=f"field {f}")
    r.adjoint(z["res_vx"], z["res_vy"], None)
    for f in (7, 8, 9):
        np.testing.assert_array_equal(r.field(f), z[f"field{f}"], err_msg=f"accumulator {f}")
    for a, n in zip(r.gradient(), ("gvp", "gvs", "grho")):
        np.testing.assert_array_equal(a, z[n], err_msg=n)


@pytest.mark.skipif(not O.reference_available(), reason="reference build not present")
def test_live_reference_forward_matches_restatement():
    p, model, src, rec, z = load("visco_l3_fd8_fs")
    p = p.replace(nt=120)
    vx, vy = O.run_isolated(O.reference_forward_sections, p, model, src[:3] + (src[3], src[4]),
                            rec)
    r = O.Restatement(p, model, (src[0], src[1], src[2][:, :120], src[3], src[4]), rec, "f")
    r.forward()
    np.testing.assert_array_equal(r.sections(0), vx)
    np.testing.assert_array_equal(r.sections(1), vy)


@pytest.mark.parametrize("name", ["elastic_fd8_fs", "visco_l3_fd8_fs"])
def test_fp32_scheme_error_against_fp64(name):
    """FP32 rounding error of the reference scheme (float restatement vs double)."""
    p, model, src, rec, z = load(name)
    rf = O.Restatement(p, model, src, rec, "f")
    rd = O.Restatement(p, model, src, rec, "d")
    rf.forward(store=True)
    rd.forward(store=True)
    e_sec = max(O.rel_l2(rf.sections(c), rd.sections(c)) for c in (0, 1))
    assert e_sec < 1e-5, e_sec
    rf.adjoint(z["res_vx"], z["res_vy"], None)
    rd.adjoint(z["res_vx"], z["res_vy"], None)
    e_grad = max(O.rel_l2(a, b) for a, b in zip(rf.gradient(), rd.gradient()))
    assert e_grad < 1e-4, e_grad
