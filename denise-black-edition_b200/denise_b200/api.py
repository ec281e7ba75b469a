"""Python mirror of the reference's P-SV operator interface over the C ABI.

The reference exposes its propagator as ``psv(..., mode)`` (src/PSV/psv.c:17)
driven by FD_PSV (forward modelling) and grad_obj_psv (per-shot gradient).
Here a :class:`Model` holds the device-resident material coefficients of one
grid, a :class:`Shot` the wavefield state and acquisition of one source, and
:func:`run` advances any number of shots through the whole time loop in one
batched launch per operation.  Arrays follow the reference's file order:
models and gradients have shape (nx, ny) (x-major, z contiguous), sections
shape (ntr, nt).
"""
import ctypes
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import check, fptr, iptr, lib


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and a.shape != tuple(shape):
        a = a.reshape(shape)
    return a


@dataclass
class PsvParams:
    """The read_par.c globals the P-SV path reads (names lower-cased)."""
    nx: int
    ny: int
    dh: float
    dt: float
    nt: int
    fdorder: int = 8
    maxrelerror: int = 1
    free_surf: int = 1
    fw: int = 20
    damping: float = 1500.0
    fpml: float = 10.0
    npower: float = 4.0
    k_max_pml: float = 1.0
    boundary: int = 0
    L: int = 0
    fl: Sequence[float] = field(default_factory=tuple)
    ts: float = 0.1
    invmat1: int = 1
    grad_form: int = 1
    quelltypb: int = 1
    seismo: int = 1
    dtinv: int = 1
    eprecond: int = 0
    store_snapshots: int = 0
    snap_precision: int = _lib.SNAP_F32
    grad_accum: int = _lib.ACC_F32
    arith: int = _lib.ARITH_EXACT
    honor_q: int = 0
    ckpt_steps: int = 0

    def to_c(self):
        p = _lib.Params()
        for name, _ in _lib.Params._fields_:
            if name == "fl":
                arr = (ctypes.c_float * _lib.DN_MAX_L)(*([0.0] * _lib.DN_MAX_L))
                for k, v in enumerate(self.fl):
                    arr[k] = float(v)
                p.fl = arr
            else:
                setattr(p, name, getattr(self, name))
        return p

    def replace(self, **kw):
        d = dict(self.__dict__)
        d.update(kw)
        return PsvParams(**d)

    @property
    def cells(self):
        return self.nx * self.ny


# ---------------------------------------------------------------------------
# host set-up numerics (bit-identical to the reference)
# ---------------------------------------------------------------------------
def holbergcoeff(fdorder, maxrelerror):
    hc = np.zeros(7, np.float32)
    check(lib.dn_holbergcoeff(fdorder, maxrelerror, fptr(hc)))
    return hc


def pml_profiles(params: PsvParams):
    """dict of the 20 CPML vectors (each 2*FW floats) of PML_pro()."""
    w = 2 * max(params.fw, 1)
    out = {n: np.zeros(w, np.float32) for n in _lib.PML_NAMES}
    pml = _lib.Pml(*[fptr(out[n]) for n in _lib.PML_NAMES])
    p = params.to_c()
    check(lib.dn_pml_profiles(ctypes.byref(p), ctypes.byref(pml)))
    return out


def average_materials(params: PsvParams, vp, vs, rho):
    shp = (params.nx, params.ny)
    vp, vs, rho = _f32(vp, shp), _f32(vs, shp), _f32(rho, shp)
    uipjp, rip, rjp = (np.zeros(shp, np.float32) for _ in range(3))
    p = params.to_c()
    check(lib.dn_average_materials(ctypes.byref(p), fptr(vp), fptr(vs), fptr(rho), fptr(uipjp), fptr(rip), fptr(rjp)))
    return {"uipjp": uipjp, "rip": rip, "rjp": rjp}


def prepare_visc(params: PsvParams, vp, vs, rho, qp=None, qs=None):
    shp = (params.nx, params.ny)
    L = params.L
    args = [_f32(a, shp) if a is not None else None for a in (vp, vs, rho, qp, qs)]
    out = {k: np.zeros(shp, np.float32) for k in ("fipjp", "f", "g")}
    out.update({k: np.zeros((L,) + shp, np.float32) for k in ("dip", "d", "e")})
    out.update({k: np.zeros(L, np.float32) for k in ("bip", "bjm", "cip", "cjm", "eta")})
    p = params.to_c()
    order = ("fipjp", "f", "g", "dip", "d", "e", "bip", "bjm", "cip", "cjm", "eta")
    check(lib.dn_prepare_visc(ctypes.byref(p), *[fptr(a) for a in args], *[fptr(out[k]) for k in order]))
    return out


def wavelet(quellart, nt, dt, tshift, fc, amp, n_order=0, fc_spike_1=0.0, fc_spike_2=0.0, ts=0.0, signal=None):
    """wavelet.c for one source.  QUELLART 3 takes `signal` (the samples of the
    wavelet file, at least nt), 7 the chirp band FC_SPIKE_1..FC_SPIKE_2 over TS;
    the spike of 6 comes unfiltered (band-limit it with tdfilt)."""
    out = np.zeros(nt, np.float32)
    sig = None if signal is None else np.ascontiguousarray(signal, np.float32)
    check(lib.dn_wavelet_ex(int(quellart), int(nt), ctypes.c_float(dt), ctypes.c_float(tshift), ctypes.c_float(fc),
                            ctypes.c_float(amp), int(n_order), ctypes.c_float(fc_spike_1), ctypes.c_float(fc_spike_2),
                            ctypes.c_float(ts), None if sig is None else fptr(sig), 0 if sig is None else sig.size,
                            fptr(out)))
    return out


def cfl_limit(params: PsvParams, vp_max):
    ds = ctypes.c_double(0.0)
    p = params.to_c()
    st = lib.dn_cfl_check(ctypes.byref(p), float(vp_max), ctypes.byref(ds))
    return ds.value, st == _lib.DN_OK


def model_footprint(params: PsvParams):
    b = ctypes.c_size_t(0)
    p = params.to_c()
    check(lib.dn_model_footprint(ctypes.byref(p), ctypes.byref(b)))
    return b.value


def device_memory(device=0):
    """(free, total) bytes of a device; free counts the blocks the library keeps cached."""
    free, total = ctypes.c_size_t(0), ctypes.c_size_t(0)
    check(lib.dn_device_memory(int(device), ctypes.byref(free), ctypes.byref(total)))
    return free.value, total.value


def device_trim(device=0):
    """Frees the device blocks the library keeps cached for reuse."""
    check(lib.dn_device_trim(int(device)))


def shot_footprint(params: PsvParams, ntr, store):
    b = ctypes.c_size_t(0)
    p = params.to_c()
    check(lib.dn_shot_footprint(ctypes.byref(p), int(ntr), int(store), ctypes.byref(b)))
    return b.value


# ---------------------------------------------------------------------------
# device objects
# ---------------------------------------------------------------------------
class Model:
    """Device-resident material coefficients of one grid (readmod + av_* + CPML)."""

    def __init__(self, params: PsvParams, vp, vs, rho, qp=None, qs=None, device=0):
        self.params = params
        shp = (params.nx, params.ny)
        self._arrays = [_f32(a, shp) if a is not None else None for a in (vp, vs, rho, qp, qs)]
        self._c = params.to_c()
        h = ctypes.c_void_p()
        check(lib.dn_model_create(ctypes.byref(self._c), *[fptr(a) for a in self._arrays], int(device),
                                  ctypes.byref(h)))
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            lib.dn_model_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def gradient(self):
        shp = (self.params.nx, self.params.ny)
        g = [np.zeros(shp, np.float32) for _ in range(3)]
        check(lib.dn_model_get_gradient(self.handle, *[fptr(a) for a in g]))
        return tuple(g)

    MATERIALS = ("rip", "rjp", "uipjp", "mu", "lam", "rho", "vp", "vs", "muss", "lamss",
                 "c_muipjp", "c_tausipjp", "c_mu", "c_taus", "c_pi", "c_taup")

    def material(self, which):
        """A material plane the kernels use (name from MATERIALS or its index), (nx, ny) file order."""
        k = self.MATERIALS.index(which) if isinstance(which, str) else int(which)
        out = np.empty((self.params.nx, self.params.ny), np.float32)
        check(lib.dn_model_get_material(self.handle, k, fptr(out)))
        return out

    def zero_gradient(self):
        check(lib.dn_model_zero_gradient(self.handle))

    def set_gradient(self, g_vp=None, g_vs=None, g_rho=None):
        """Replaces the stacked gradients (file order (nx, ny) arrays; None keeps a class)."""
        arrs = [None if g is None else np.ascontiguousarray(g, np.float32) for g in (g_vp, g_vs, g_rho)]
        check(lib.dn_model_set_gradient(self.handle, *[fptr(a) for a in arrs]))


class Shot:
    """Wavefield state + acquisition of one shot on a model's device."""

    def __init__(self, model: Model, src_i, src_j, signals, rec_i, rec_j, src_type=None, src_azi=None):
        self.model = model
        p = model.params
        self.src_i = np.ascontiguousarray(src_i, np.int32)
        self.src_j = np.ascontiguousarray(src_j, np.int32)
        self.nsrc = len(self.src_i)
        self.signals = _f32(signals, (self.nsrc, p.nt))
        self.src_type = np.ascontiguousarray(src_type if src_type is not None else np.ones(self.nsrc), np.int32)
        self.src_azi = _f32(src_azi if src_azi is not None else np.zeros(self.nsrc))
        self.rec_i = np.ascontiguousarray(rec_i, np.int32)
        self.rec_j = np.ascontiguousarray(rec_j, np.int32)
        self.ntr = len(self.rec_i)
        acq = _lib.Acq(self.nsrc, iptr(self.src_i), iptr(self.src_j), iptr(self.src_type), fptr(self.src_azi),
                       fptr(self.signals), self.ntr, iptr(self.rec_i), iptr(self.rec_j))
        h = ctypes.c_void_p()
        check(lib.dn_shot_create(model.handle, ctypes.byref(acq), ctypes.byref(h)))
        self.handle = h

    def close(self):
        if self.handle:
            lib.dn_shot_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sections(self, comp=_lib.SEC_VX):
        out = np.empty((self.ntr, self.model.params.nt), np.float32)
        check(lib.dn_shot_get_sections(self.handle, comp, fptr(out)))
        return out

    def set_residuals(self, vx=None, vy=None, p=None):
        shp = (self.ntr, self.model.params.nt)
        arrs = [_f32(a, shp) if a is not None else None for a in (vx, vy, p)]
        check(lib.dn_shot_set_residuals(self.handle, *[fptr(a) for a in arrs]))

    def residual(self, obs, comp=_lib.SEC_VX):
        """L2 residual against observed data obs (ntr, nt) into this shot's adjoint
        source of `comp`; returns the component's misfit 0.5*sum(r^2)."""
        l2 = ctypes.c_double(0.0)
        o = _f32(obs, (self.ntr, self.model.params.nt))
        check(lib.dn_shot_residual(self.handle, comp, fptr(o), ctypes.byref(l2)))
        return l2.value

    def residual_ex(self, obs, comp=_lib.SEC_VX, **opts):
        """calc_res with the options of dn_residual_opts (lnorm, grad_form, mode, n_order,
        comp_weight, c_vp, c_rho, fc_start, fc_end, kill, offset_mute, offsetc, timewin,
        gamma, twlength_minus, src_x, src_z); stores the residual as this component's
        adjoint source and returns the misfit."""
        o, keep = residual_opts(**opts)
        obs = np.ascontiguousarray(obs, np.float32)
        out = ctypes.c_double()
        check(lib.dn_shot_residual_ex(self.handle, comp, fptr(obs), ctypes.byref(o), ctypes.byref(out)))
        return out.value

    def rtm_source(self, obs, comp=_lib.SEC_VX):
        """Reverse-time-migration source (calc_res MODE 2): the observed data
        itself, time-reversed and integrated, as this shot's adjoint source."""
        o = _f32(obs, (self.ntr, self.model.params.nt))
        check(lib.dn_shot_rtm_source(self.handle, comp, fptr(o)))

    def accumulate_gradient(self):
        check(lib.dn_shot_accumulate_gradient(self.handle))

    def accumulate_gradient_precond(self, c_vp, c_vs, c_rho):
        """ass_gradPSV with the per-shot energy preconditioning (EPRECOND 1 or 3)."""
        check(lib.dn_shot_accumulate_gradient_precond(self.handle, float(c_vp), float(c_vs), float(c_rho)))

    def accumulate_gradient_ex(self, energy=None, circular_taper=None):
        """Gradient assembly with the per-shot options of grad_obj_psv.c:214-250.
        energy = (c_vp, c_vs, c_rho) for EPRECOND 1/3 scaling; circular_taper =
        (srtshape, srtradius, filtsize, src_x, src_z) for taper_grad_shot around
        this shot's source (metres)."""
        o = _lib.AccumOpts()
        if energy is not None:
            o.energy = 1
            o.c_vp, o.c_vs, o.c_rho = (float(x) for x in energy)
        if circular_taper is not None:
            o.circular_taper = 1
            o.srtshape, o.srtradius, o.filtsize, o.src_x, o.src_z = circular_taper
        check(lib.dn_shot_accumulate_gradient_ex(self.handle, ctypes.byref(o)))

    def field(self, fid):
        out = np.zeros((self.model.params.nx, self.model.params.ny), np.float32)
        check(lib.dn_shot_get_field(self.handle, fid, fptr(out)))
        return out

    def snapshot(self, k, f):
        out = np.zeros((self.model.params.nx, self.model.params.ny), np.float32)
        check(lib.dn_shot_get_snapshot(self.handle, k, f, fptr(out)))
        return out

    def run_steps(self, mode, nt0, nt1):
        check(lib.dn_run_steps(self.handle, mode, nt0, nt1))

    def kernel(self):
        """(kernel variant, whether forward runs take the fused elastic step)"""
        v, f = ctypes.c_int(), ctypes.c_int()
        check(lib.dn_shot_kernel(self.handle, ctypes.byref(v), ctypes.byref(f)))
        return v.value, bool(f.value)


def tdfilt(traces, dt, order, fc_low, fc_high=0.0, device=0):
    """apply_tdfilt: Butterworth low-pass at fc_low, then high-pass at fc_high if > 0, of
    [ntr][ns] traces (host array; a filtered copy is returned)."""
    a = np.array(traces, np.float32, copy=True, order="C")
    two_d = a.ndim == 2
    a = a.reshape(-1, a.shape[-1])
    check(lib.dn_tdfilt_host(fptr(a), a.shape[0], a.shape[1], ctypes.c_float(dt), int(order),
                             ctypes.c_float(fc_low), ctypes.c_float(fc_high), int(device)))
    return a if two_d else a.reshape(-1)


def residual_opts(lnorm=2, grad_form=1, mode=1, n_order=0, comp_weight=0, c_vp=0.0, c_rho=0.0, fc_start=0.0,
                  fc_end=0.0, kill=None, offset_mute=0, offsetc=0.0, timewin=0, gamma=0.0, twlength_minus=1.0,
                  src_x=0.0, src_z=0.0):
    """dn_residual_opts and the arrays it points to (keep both alive)."""
    o = _lib.ResidualOpts(lnorm=lnorm, grad_form=grad_form, mode=mode, n_order=n_order, comp_weight=comp_weight,
                          c_vp=c_vp, c_rho=c_rho, fc_start=fc_start, fc_end=fc_end, offset_mute=offset_mute,
                          offsetc=offsetc, timewin=timewin, gamma=gamma, twlength_minus=twlength_minus, src_x=src_x,
                          src_z=src_z)
    keep = None
    if kill is not None:
        keep = np.ascontiguousarray(kill, np.int32)
        o.kill = iptr(keep)
    return o, keep


FIELDS = {"vx": 0, "vy": 1, "sxx": 2, "syy": 3, "sxy": 4, "vxp1": 5, "vyp1": 6,
          "waveconv_shot": 7, "waveconv_u_shot": 8, "waveconv_rho_shot": 9, "Ws": 10, "Wr": 11}


def run(shots: Sequence[Shot], mode=_lib.MODE_FORWARD):
    """Whole time loop for a batch of shots (one launch per operation, graph-replayed)."""
    arr = (ctypes.c_void_p * len(shots))(*[s.handle for s in shots])
    check(lib.dn_run(arr, len(shots), mode))


def run_plain(shot: Shot, mode=_lib.MODE_FORWARD):
    """One shot, direct launches per time step (the un-batched path)."""
    check(lib.dn_run_plain(shot.handle, mode))


def last_run_stats():
    ms = ctypes.c_double(0.0)
    nl = ctypes.c_longlong(0)
    lib.dn_last_run_stats(ctypes.byref(ms), ctypes.byref(nl))
    return ms.value, nl.value


KERNEL_SLOTS = ("update_v", "inject_v", "update_s", "inject_s", "surface", "seismo", "snap_store", "correlate")


def profile_steps(shots: Sequence[Shot], mode=_lib.MODE_FORWARD, nsteps=20):
    """Average device ms per launch of each kernel of the batched step."""
    arr = (ctypes.c_void_p * len(shots))(*[s.handle for s in shots])
    out = (ctypes.c_double * 8)()
    check(lib.dn_profile_steps(arr, len(shots), mode, nsteps, out))
    return dict(zip(KERNEL_SLOTS, list(out)))
