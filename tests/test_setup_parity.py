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


# (QUELLART, n_order, tshift, fc, amp, fc_spike_1, fc_spike_2, ts)
WAVELETS = [(1, 0, 0.01, 12.0, 2.5, 0, 0, 0), (1, 2, 0.0, 30.0, 1.0, 0, 0, 0), (2, 0, 0.004, 40.0, 1.0, 0, 0, 0),
            (4, 1, 0.002, 25.0, 3.0, 0, 0, 0), (5, 0, 0.0, 18.0, 1.0, 0, 0, 0), (6, 0, 0.0135, 10.0, 7.0, 0, 0, 0),
            (6, 1, 0.0, 10.0, 1.0, 0, 0, 0), (7, 0, 0.003, 10.0, 2.0, 7.0, 45.0, 0.04),
            (7, 1, 0.0, 10.0, 1.0, 12.0, 60.0, 0.03), (3, 0, 0.0, 10.0, 1.5, 0, 0, 0), (3, 2, 0.0, 10.0, 1.0, 0, 0, 0)]


@pytest.mark.skipif(not O.reference_available(), reason="reference build not present")
@pytest.mark.parametrize("w", WAVELETS, ids=lambda w: f"q{w[0]}-n{w[1]}-t{w[2]}")
def test_wavelets_match_live_reference(tmp_path, w):
    """dn_wavelet_ex against the reference's wavelet() with every global it reads
    set: all seven QUELLART, time shifts on and off the sample grid, N_ORDER
    integrations, the Klauder chirp band and the wavelet file of QUELLART 3."""
    qa, n_order, tshift, fc, amp, f1, f2, ts = w
    nt, dt = 700, 2.5e-4
    signal = None
    if qa == 3:
        rng = np.random.default_rng(7)
        signal = np.cumsum(rng.standard_normal(nt + 5)).astype(np.float32)
    want = O.run_isolated(O.ref_wavelet_ex, str(tmp_path), qa, n_order, nt, dt, tshift, fc, amp, f1, f2, ts, signal)
    if qa == 3:   # what the reference read back from the text file
        from denise_b200 import io

        signal = io.read_signal_file(str(tmp_path / "sig_shot_1.dat"))
        assert signal.size == nt + 5
    got = dn.wavelet(qa, nt, dt, tshift, fc, amp, n_order, fc_spike_1=f1, fc_spike_2=f2, ts=ts, signal=signal)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_wavelet_file_shorter_than_nt_is_rejected():
    """A wavelet file with fewer samples than NT is an error (the reference would
    read past its buffer); dn_wavelet asks for dn_wavelet_ex for QUELLART 3 and 7."""
    import ctypes

    from denise_b200 import _lib

    with pytest.raises(dn.DeniseError, match="DN_EINVAL"):
        dn.wavelet(3, 100, 1e-3, 0.0, 10.0, 1.0, signal=np.zeros(99, np.float32))
    out = np.zeros(100, np.float32)
    for qa in (3, 7):
        with pytest.raises(dn.DeniseError, match="DN_EINVAL"):
            _lib.check(_lib.lib.dn_wavelet(qa, 100, ctypes.c_float(1e-3), ctypes.c_float(0.0), ctypes.c_float(10.0),
                                           ctypes.c_float(1.0), 0, out.ctypes.data_as(_lib._c_float_p)))
