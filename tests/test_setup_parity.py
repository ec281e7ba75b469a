"""Host set-up numerics of the product library against the reference (no GPU).

dn_holbergcoeff / dn_pml_profiles / dn_average_materials / dn_prepare_visc /
dn_wavelet are compared bit for bit with the reference's own outputs stored in
tests/golden/ and, when the reference build is present, with live runs over
further parameter sets (CPML width, npower, damping, FPML, Q, L).
"""
import numpy as np
import pytest

import denise_b200 as dn
from denise_b200 import synth
from denise_b200._lib import PML_NAMES

import oracles as O
from golden.make_golden import CASES, load


def _pml_flat(p):
    pm = dn.pml_profiles(p)
    return np.concatenate([pm[n] for n in PML_NAMES])


@pytest.mark.parametrize("name", sorted(CASES))
def test_setup_matches_reference_golden(name):
    p, model, src, rec, z = load(name)
    np.testing.assert_array_equal(dn.holbergcoeff(p.fdorder, p.maxrelerror), z["hc"])
    np.testing.assert_array_equal(_pml_flat(p), z["pml"])
    am = dn.average_materials(p, *model[:3])
    for n in ("rip", "rjp", "uipjp"):
        np.testing.assert_array_equal(am[n], z[n], err_msg=n)
    if p.L:
        pv = dn.prepare_visc(p, *model)
        for n in ("fipjp", "f", "g", "dip", "d", "e"):
            np.testing.assert_array_equal(pv[n], z[n], err_msg=n)
        vv = np.stack([pv["bip"], pv["bjm"], pv["cip"], pv["cjm"], pv["eta"]])
        np.testing.assert_array_equal(vv, z["visc_vectors"])
    for qa in (1, 2, 4, 5, 6):
        np.testing.assert_array_equal(dn.wavelet(qa, p.nt, p.dt, 0.0, 25.0, 1.5), z[f"wavelet{qa}"],
                                      err_msg=f"QUELLART {qa}")


def test_holberg_table_matches_restatement():
    for fo in (2, 4, 6, 8, 10, 12):
        for e in range(5):
            p = synth.c0_params(nx=24, ny=24, nt=4, fw=4, fdorder=fo, maxrelerror=e)
            z = np.zeros((24, 24), np.float32) + 2000
            r = O.Restatement(p, (z, z / 2, z / 2), (np.array([5], np.int32), np.array([5], np.int32),
                                                     np.zeros((1, 4), np.float32)), (np.array([3], np.int32),
                                                                                       np.array([3], np.int32)))
            np.testing.assert_array_equal(dn.holbergcoeff(fo, e), r.setup(0))


def test_bad_fd_parameters_are_rejected():
    with pytest.raises(dn.DeniseError) as e:
        dn.holbergcoeff(7, 1)
    assert e.value.code == -1
    with pytest.raises(dn.DeniseError):
        dn.holbergcoeff(8, 5)


def _live_setup(p, model):
    src = (np.array([p.nx // 2], np.int32), np.array([3], np.int32), np.zeros((1, p.nt), np.float32))
    rec = (np.array([5], np.int32), np.array([4], np.int32))
    r = O.Reference(p, model, src, rec, mode_global=0)
    out = {"pml": r.pml(), "rip": r.mat(0), "rjp": r.mat(1), "uipjp": r.mat(2)}
    if p.L:
        out["fipjp"] = r.mat(3)
        out["d1"] = r.mat(201)
    return out


PML_SETS = [dict(fw=20, damping=1500.0, fpml=10.0, npower=4.0, k_max_pml=1.0),
            dict(fw=7, damping=3000.0, fpml=25.0, npower=2.0, k_max_pml=1.0),
            dict(fw=15, damping=800.0, fpml=5.0, npower=3.0, k_max_pml=2.5, dh=2.5, dt=2e-4)]


@pytest.mark.skipif(not O.reference_available(), reason="reference build not present")
@pytest.mark.parametrize("kw", PML_SETS, ids=["default", "thin", "kmax"])
def test_setup_matches_live_reference(kw):
    p = synth.c0_params(nx=70, ny=52, nt=10, L=2, fl=(3.0, 20.0), **kw)
    vp, vs, rho = synth.base_model(p.nx, p.ny, p.dh, 9)
    vs[:5, :3] = 0.0            # zero-shear corner: uipjp -> 0 (av_mue.c:40)
    rho[-3:, -2:] = 5e-5        # near-zero density: rip/rjp -> 0 (av_rho.c:17-22)
    qp, qs = synth.q_model(p.nx, p.ny, 9)
    R = O.run_isolated(_live_setup, p, (vp, vs, rho, qp, qs))
    np.testing.assert_array_equal(_pml_flat(p), R["pml"])
    am = dn.average_materials(p, vp, vs, rho)
    for n in ("rip", "rjp", "uipjp"):
        np.testing.assert_array_equal(am[n], R[n], err_msg=n)
    pv = dn.prepare_visc(p, vp, vs, rho, qp, qs)
    np.testing.assert_array_equal(pv["fipjp"], R["fipjp"])
    np.testing.assert_array_equal(pv["d"][0], R["d1"])
