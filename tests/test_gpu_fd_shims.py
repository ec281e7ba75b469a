"""Per-kernel drop-ins with the reference's own signatures (libdenise_b200_fd.so):
update_v_PML_PSV, update_s_elastic_PML_PSV and update_s_visc_PML_PSV called the way psv() calls the
reference's functions, on NR-style arrays (matrix() blocks with their halos),
side by side with the reference's own functions from its build: the updated
fields, vxp1 / vyp1, the CPML memory and the QUELLTYP the velocity update leaves
are bit-identical, for FDORDER 2-12, free surface on and off, forward (sw 0,
force sources of every type, two in one cell) and adjoint (sw 1, QUELLTYPB)
calls, INVMAT1 1 and 3 for the elastic stress update, and L = 1..5 memory
variables for the viscoelastic one (its prepared fipjp, f, g, d, e, dip)."""
import ctypes
import os

import numpy as np
import pytest

from denise_b200 import _lib

import oracles as O

pytestmark = pytest.mark.gpu

SHIM = os.path.join(os.path.dirname(_lib.LIB_PATH), "libdenise_b200_fd.so")


class NR:
    """matrix(nrl, nrh, ncl, nch) of the reference: one float32 block and its row
    pointers; `.ptr` is the float** the reference indexes from (nrl, ncl)."""

    def __init__(self, nrl, nrh, ncl, nch, data):
        self.a = np.ascontiguousarray(data, np.float32).copy()
        assert self.a.shape == (nrh - nrl + 1, nch - ncl + 1)
        base, nc = self.a.ctypes.data, self.a.shape[1]
        self.rows = (ctypes.c_void_p * self.a.shape[0])(*[base + (r * nc - ncl) * 4 for r in range(self.a.shape[0])])
        self.ptr = ctypes.c_void_p(ctypes.addressof(self.rows) - nrl * 8)


class T3:
    """f3tensor(nrl, nrh, ncl, nch, ndl, ndh) of the reference: one float32 block
    [row][col][depth] and two levels of pointers; `.ptr` is the float***."""

    def __init__(self, nrl, nrh, ncl, nch, ndl, ndh, data):
        self.a = np.ascontiguousarray(data, np.float32).copy()
        nr, nc, nd = self.a.shape
        assert (nr, nc, nd) == (nrh - nrl + 1, nch - ncl + 1, ndh - ndl + 1)
        base = self.a.ctypes.data
        self.cols = [(ctypes.c_void_p * nc)(*[base + ((r * nc + c) * nd - ndl) * 4 for c in range(nc)])
                     for r in range(nr)]
        self.rows = (ctypes.c_void_p * nr)(*[ctypes.addressof(cl) - ncl * 8 for cl in self.cols])
        self.ptr = ctypes.c_void_p(ctypes.addressof(self.rows) - nrl * 8)


class Vec:
    """vector(1, n) of the reference."""

    def __init__(self, data):
        self.a = np.ascontiguousarray(data, np.float32).copy()
        self.ptr = ctypes.c_void_p(self.a.ctypes.data - 4)


def _libs():
    if not O.reference_available():
        pytest.skip("the reference build (oracle/_ref) is not there")
    ref = ctypes.CDLL(O.REF_SO, mode=ctypes.RTLD_GLOBAL)   # its globals resolve the shim's references
    return ref, ctypes.CDLL(SHIM)


def _globals(ref, nx, ny, fdorder, fw, free_surf, nt_total, quelltypb=1, invmat1=1, L=0):
    ints = dict(NX=nx, NY=ny, FDORDER=fdorder, FW=fw, FREE_SURF=free_surf, BOUNDARY=0, NPROCX=1, NPROCY=1,
                GRAD_FORM=1, INVMAT1=invmat1, NT=nt_total, QUELLTYPB=quelltypb, MYID=0, QUELLTYP=0, L=L)
    for k, v in ints.items():
        ctypes.c_int.in_dll(ref, k).value = v
    ctypes.c_float.in_dll(ref, "DT").value = 4e-4
    ctypes.c_float.in_dll(ref, "DH").value = 5.0
    pos = (ctypes.c_int * 3).in_dll(ref, "POS")
    pos[0] = pos[1] = pos[2] = 0


@pytest.mark.parametrize("sw", [0, 1])
@pytest.mark.parametrize("fdorder,free_surf", [(2, 1), (4, 0), (6, 1), (8, 1), (8, 0), (10, 0), (12, 1)])
def test_update_v_matches_reference(fdorder, free_surf, sw):
    ref, shim = _libs()
    nx, ny, fw, nt_total, nt = 61, 37, 10, 20, 7
    _globals(ref, nx, ny, fdorder, fw, free_surf, nt_total, quelltypb=1 if fdorder % 4 else 3)
    rng = np.random.default_rng(fdorder * 10 + sw)
    nd = fdorder // 2 + 1
    fshape = (ny + 2 * nd, nx + 2 * nd)
    fb = (-nd + 1, ny + nd, -nd + 1, nx + nd)
    fields = {k: rng.standard_normal(fshape).astype(np.float32) for k in
              ("vx", "vy", "sxx", "syy", "sxy", "vxp1", "vyp1", "vxm1", "vym1", "uttx", "utty", "absorb")}
    mats = {k: (1e-3 * (0.5 + rng.random(fshape))).astype(np.float32) for k in ("rip", "rjp")}
    psis = {"psi_sxx_x": rng.standard_normal((ny, 2 * fw)), "psi_sxy_x": rng.standard_normal((ny, 2 * fw)),
            "psi_syy_y": rng.standard_normal((2 * fw, nx)), "psi_sxy_y": rng.standard_normal((2 * fw, nx))}
    nsrc = 4
    src = np.zeros((8, nsrc), np.float32)
    src[0] = [5, 30, 30, 61]            # i (the last one on the right edge)
    src[1] = [3, 20, 20, 37]            # j; two sources share (30, 20)
    src[6] = [0.0, 35.0, 120.0, 0.0]    # azimuth
    src[7] = [2, 4, 3, 4]               # QUELLTYP of each
    sig = rng.standard_normal((nsrc, nt_total)).astype(np.float32)
    sig1 = rng.standard_normal((nsrc, nt_total)).astype(np.float32)
    hc = Vec(rng.standard_normal(fdorder // 2))
    cp = [Vec(1.0 + rng.random(2 * fw)), Vec(-0.2 * rng.random(2 * fw)), Vec(0.5 + 0.5 * rng.random(2 * fw))]
    cpml = [Vec(cp[k % 3].a * (1.0 + 0.01 * (k // 3))) for k in range(12)]
    out = {}
    for name, lib in (("ref", ref), ("shim", shim)):
        F = {k: NR(*fb, v) for k, v in fields.items()}
        M = {k: NR(*fb, v) for k, v in mats.items()}
        P = {k: NR(1, v.shape[0], 1, v.shape[1], v) for k, v in psis.items()}
        S, G, G1 = NR(1, 8, 1, nsrc, src), NR(1, nsrc, 1, nt_total, sig), NR(1, nsrc, 1, nt_total, sig1)
        ctypes.c_int.in_dll(ref, "QUELLTYP").value = 0
        lib.update_v_PML_PSV(1, nx, 1, ny, nt, F["vx"].ptr, F["vxp1"].ptr, F["vxm1"].ptr, F["vy"].ptr, F["vyp1"].ptr,
                             F["vym1"].ptr, F["uttx"].ptr, F["utty"].ptr, F["sxx"].ptr, F["syy"].ptr, F["sxy"].ptr,
                             M["rip"].ptr, M["rjp"].ptr, S.ptr, G.ptr, G1.ptr, nsrc, F["absorb"].ptr, hc.ptr, 0, sw,
                             *[v.ptr for v in cpml], P["psi_sxx_x"].ptr, P["psi_syy_y"].ptr, P["psi_sxy_y"].ptr,
                             P["psi_sxy_x"].ptr)
        out[name] = ({k: F[k].a for k in ("vx", "vy", "vxp1", "vyp1", "sxx")}, {k: P[k].a for k in P},
                     ctypes.c_int.in_dll(ref, "QUELLTYP").value)
    for k in out["ref"][0]:
        np.testing.assert_array_equal(out["shim"][0][k], out["ref"][0][k], err_msg=k)
    for k in out["ref"][1]:
        np.testing.assert_array_equal(out["shim"][1][k], out["ref"][1][k], err_msg=k)
    assert out["shim"][2] == out["ref"][2]
    assert not np.array_equal(out["ref"][0]["vx"], fields["vx"])   # the call did update


@pytest.mark.parametrize("invmat1", [1, 3])
@pytest.mark.parametrize("fdorder,free_surf", [(2, 0), (4, 1), (8, 1), (8, 0), (12, 0)])
def test_update_s_elastic_matches_reference(fdorder, free_surf, invmat1):
    ref, shim = _libs()
    nx, ny, fw, nt_total = 61, 37, 10, 20
    _globals(ref, nx, ny, fdorder, fw, free_surf, nt_total, invmat1=invmat1)
    rng = np.random.default_rng(fdorder * 100 + invmat1)
    nd = fdorder // 2 + 1
    fshape = (ny + 2 * nd, nx + 2 * nd)
    fb = (-nd + 1, ny + nd, -nd + 1, nx + nd)
    fields = {k: rng.standard_normal(fshape).astype(np.float32) for k in
              ("vx", "vy", "sxx", "syy", "sxy", "ux", "uy", "uxy", "uyx", "absorb")}
    mats = {"pi": 2000 + 2000 * rng.random(fshape), "u": 1000 + 1000 * rng.random(fshape),
            "rho": 2000 + 500 * rng.random(fshape), "uipjp": 1e9 * (1 + rng.random(fshape))}
    if invmat1 == 3:
        mats["pi"], mats["u"] = 1e10 * (1 + rng.random(fshape)), 5e9 * (1 + rng.random(fshape))
    psis = {"psi_vxx": rng.standard_normal((ny, 2 * fw)), "psi_vyx": rng.standard_normal((ny, 2 * fw)),
            "psi_vyy": rng.standard_normal((2 * fw, nx)), "psi_vxy": rng.standard_normal((2 * fw, nx))}
    hc = Vec(rng.standard_normal(fdorder // 2))
    cp = [Vec(1.0 + rng.random(2 * fw)), Vec(-0.2 * rng.random(2 * fw)), Vec(0.5 + 0.5 * rng.random(2 * fw))]
    cpml = [Vec(cp[k % 3].a * (1.0 + 0.01 * (k // 3))) for k in range(12)]
    out = {}
    for name, lib in (("ref", ref), ("shim", shim)):
        F = {k: NR(*fb, v) for k, v in fields.items()}
        M = {k: NR(*fb, v) for k, v in mats.items()}
        P = {k: NR(1, v.shape[0], 1, v.shape[1], v) for k, v in psis.items()}
        lib.update_s_elastic_PML_PSV(1, nx, 1, ny, F["vx"].ptr, F["vy"].ptr, F["ux"].ptr, F["uy"].ptr, F["uxy"].ptr,
                                     F["uyx"].ptr, F["sxx"].ptr, F["syy"].ptr, F["sxy"].ptr, M["pi"].ptr, M["u"].ptr,
                                     M["uipjp"].ptr, F["absorb"].ptr, M["rho"].ptr, hc.ptr, 0,
                                     *[v.ptr for v in cpml], P["psi_vxx"].ptr, P["psi_vyy"].ptr, P["psi_vxy"].ptr,
                                     P["psi_vyx"].ptr, 0)
        out[name] = ({k: F[k].a for k in ("sxx", "syy", "sxy", "vx")}, {k: P[k].a for k in P})
    for k in out["ref"][0]:
        np.testing.assert_array_equal(out["shim"][0][k], out["ref"][0][k], err_msg=k)
    for k in out["ref"][1]:
        np.testing.assert_array_equal(out["shim"][1][k], out["ref"][1][k], err_msg=k)
    assert not np.array_equal(out["ref"][0]["sxx"], fields["sxx"])


@pytest.mark.parametrize("L", [1, 3, 5])
@pytest.mark.parametrize("fdorder,free_surf", [(4, 1), (8, 0), (8, 1), (12, 0)])
def test_update_s_visc_matches_reference(fdorder, free_surf, L):
    ref, shim = _libs()
    nx, ny, fw, nt_total = 61, 37, 10, 20
    _globals(ref, nx, ny, fdorder, fw, free_surf, nt_total, L=L)
    rng = np.random.default_rng(fdorder * 1000 + L)
    nd = fdorder // 2 + 1
    fshape = (ny + 2 * nd, nx + 2 * nd)
    fb = (-nd + 1, ny + nd, -nd + 1, nx + nd)
    fields = {k: rng.standard_normal(fshape).astype(np.float32) for k in
              ("vx", "vy", "sxx", "syy", "sxy", "ux", "uy", "uxy", "uyx")}
    mats = {k: (1 + rng.random(fshape)).astype(np.float32) for k in ("pi", "u", "uipjp", "rho")}
    pre = {"fipjp": 1e3 * (1 + rng.random(fshape)), "f": 1e3 * (1 + rng.random(fshape)),
           "g": 1e3 * (1 + rng.random(fshape))}
    tens = {k: rng.standard_normal(fshape + (L,)) for k in ("r", "p", "q")}
    tens.update({k: 1e2 * (1 + rng.random(fshape + (L,))) for k in ("d", "e", "dip")})
    bip = (0.5 + 0.5 * rng.random(L)).astype(np.float32)
    cip = (0.5 + 0.5 * rng.random(L)).astype(np.float32)
    psis = {"psi_vxx": rng.standard_normal((ny, 2 * fw)), "psi_vyx": rng.standard_normal((ny, 2 * fw)),
            "psi_vyy": rng.standard_normal((2 * fw, nx)), "psi_vxy": rng.standard_normal((2 * fw, nx))}
    hc = Vec(rng.standard_normal(fdorder // 2))
    cp = [Vec(1.0 + rng.random(2 * fw)), Vec(-0.2 * rng.random(2 * fw)), Vec(0.5 + 0.5 * rng.random(2 * fw))]
    cpml = [Vec(cp[k % 3].a * (1.0 + 0.01 * (k // 3))) for k in range(12)]
    out = {}
    for name, lib in (("ref", ref), ("shim", shim)):
        F = {k: NR(*fb, v) for k, v in fields.items()}
        M = {k: NR(*fb, v) for k, v in mats.items()}
        Q = {k: NR(*fb, v) for k, v in pre.items()}
        T = {k: T3(*fb, 1, L, v) for k, v in tens.items()}
        P = {k: NR(1, v.shape[0], 1, v.shape[1], v) for k, v in psis.items()}
        B, Bj, C, Cj = Vec(bip), Vec(bip), Vec(cip), Vec(cip)
        lib.update_s_visc_PML_PSV(1, nx, 1, ny, F["vx"].ptr, F["vy"].ptr, F["ux"].ptr, F["uy"].ptr, F["uxy"].ptr,
                                  F["uyx"].ptr, F["sxx"].ptr, F["syy"].ptr, F["sxy"].ptr, M["pi"].ptr, M["u"].ptr,
                                  M["uipjp"].ptr, M["rho"].ptr, hc.ptr, 0, T["r"].ptr, T["p"].ptr, T["q"].ptr,
                                  Q["fipjp"].ptr, Q["f"].ptr, Q["g"].ptr, B.ptr, Bj.ptr, C.ptr, Cj.ptr, T["d"].ptr,
                                  T["e"].ptr, T["dip"].ptr, *[v.ptr for v in cpml], P["psi_vxx"].ptr,
                                  P["psi_vyy"].ptr, P["psi_vxy"].ptr, P["psi_vyx"].ptr, 0)
        out[name] = ({k: F[k].a for k in ("sxx", "syy", "sxy", "vx")}, {k: P[k].a for k in P},
                     {k: T[k].a for k in ("r", "p", "q")})
    for part in range(3):
        for k in out["ref"][part]:
            np.testing.assert_array_equal(out["shim"][part][k], out["ref"][part][k], err_msg=k)
    assert not np.array_equal(out["ref"][2]["r"], tens["r"].astype(np.float32))
