"""Host file I/O of the P-SV path (include/denise_b200_io.h) from Python:
the .inp reader, model/source/receiver files, SU output and the forward
driver.  Thin ctypes wrappers; the work is done by the C library."""
import ctypes

import numpy as np

from . import _lib
from ._lib import DN_MAX_L, Params, check, lib

DN_STR = 256


class Inp(ctypes.Structure):
    """Mirror of struct dn_inp (field for field)."""

    _fields_ = (
        [(n, ctypes.c_int) for n in ("mode", "physics", "nprocx", "nprocy", "fdorder", "maxrelerror", "nx", "ny")]
        + [(n, ctypes.c_float) for n in ("dh", "time", "dt")]
        + [("quellart", ctypes.c_int), ("signal_file", ctypes.c_char * DN_STR), ("ts", ctypes.c_float),
           ("srcrec", ctypes.c_int), ("source_file", ctypes.c_char * DN_STR), ("run_multiple_shots", ctypes.c_int),
           ("fc_spike_1", ctypes.c_float), ("fc_spike_2", ctypes.c_float),
           ("order_spike", ctypes.c_int), ("write_stf", ctypes.c_int), ("readmod", ctypes.c_int),
           ("mfile", ctypes.c_char * DN_STR), ("writemod", ctypes.c_int), ("L", ctypes.c_int),
           ("fl", ctypes.c_float * (DN_MAX_L + 1)), ("tau", ctypes.c_float),
           ("free_surf", ctypes.c_int), ("fw", ctypes.c_int)]
        + [(n, ctypes.c_float) for n in ("damping", "fpml", "npower", "k_max_pml")]
        + [(n, ctypes.c_int) for n in ("boundary", "snap", "snap_shot")]
        + [(n, ctypes.c_float) for n in ("tsnap1", "tsnap2", "tsnapinc")]
        + [(n, ctypes.c_int) for n in ("idx", "idy", "snap_format")]
        + [("snap_file", ctypes.c_char * DN_STR), ("seismo", ctypes.c_int), ("readrec", ctypes.c_int),
           ("rec_file", ctypes.c_char * DN_STR), ("refrec", ctypes.c_float * 4), ("n_streamer", ctypes.c_int),
           ("rec_incr_x", ctypes.c_float), ("rec_incr_y", ctypes.c_float), ("ndt", ctypes.c_int),
           ("seis_format", ctypes.c_int)]
        + [(n, ctypes.c_char * DN_STR) for n in ("seis_file_vx", "seis_file_vy", "seis_file_curl", "seis_file_div",
                                                  "seis_file_p", "log_file")]
        + [("log", ctypes.c_int), ("itermax", ctypes.c_int), ("jacobian", ctypes.c_char * DN_STR),
           ("data_dir", ctypes.c_char * DN_STR), ("taper", ctypes.c_int), ("taperlength", ctypes.c_int),
           ("gradt", ctypes.c_int * 5), ("invmat1", ctypes.c_int), ("grad_form", ctypes.c_int),
           ("quelltypb", ctypes.c_int), ("testshot", ctypes.c_int * 4), ("dtinv", ctypes.c_int),
           ("lnorm", ctypes.c_int), ("lines", ctypes.c_int)]
        + [(n, ctypes.c_int) for n in ("sws_taper_grad_vert", "sws_taper_grad_hor")]
        + [("exp_taper_grad_hor", ctypes.c_float)]
        + [(n, ctypes.c_int) for n in ("sws_taper_grad_sources", "sws_taper_circular_per_shot", "srtshape")]
        + [("srtradius", ctypes.c_float), ("filtsize", ctypes.c_int), ("sws_taper_file", ctypes.c_int),
           ("tfile", ctypes.c_char * DN_STR), ("inv_mod_out", ctypes.c_int), ("inv_modelfile", ctypes.c_char * DN_STR)]
        + [(n, ctypes.c_float) for n in ("vpupperlim", "vplowerlim", "vsupperlim", "vslowerlim", "rhoupperlim",
                                         "rholowerlim", "qsupperlim", "qslowerlim")]
        + [(n, ctypes.c_int) for n in ("grad_method", "pcg_beta", "nlbfgs", "model_filter", "filt_size")]
        + [("eps_scale", ctypes.c_float), ("stepmax", ctypes.c_int), ("scalefac", ctypes.c_float),
           ("trkill", ctypes.c_int)]
        + [(n, ctypes.c_char * DN_STR) for n in ("trkill_file", "picks_file", "misfit_log_file")]
        + [(n, ctypes.c_int) for n in ("min_iter", "grad_filter", "filt_size_grad", "timelapse")]
        + [("data_dir_t0", ctypes.c_char * DN_STR)]
        + [(n, ctypes.c_int) for n in ("rtmod", "gravity", "ngravb", "nzgrav", "grav_type", "back_density")]
        + [("dfile", ctypes.c_char * DN_STR), ("rtm_shot", ctypes.c_int)]
    )

    def get(self, name):
        v = getattr(self, name)
        if isinstance(v, bytes):
            return v.decode()
        if hasattr(v, "__len__"):
            return list(v)
        return v


def read_inp(path):
    inp = Inp()
    check(lib.dn_inp_read(str(path).encode(), ctypes.byref(inp)))
    return inp


def inp_nt(inp):
    return lib.dn_inp_nt(ctypes.byref(inp))


def inp_params(inp, ts):
    p = Params()
    check(lib.dn_inp_params(ctypes.byref(inp), ctypes.c_float(ts), ctypes.byref(p)))
    return p


def read_model_file(path, nx, ny):
    out = np.empty((nx, ny), np.float32)
    check(lib.dn_read_model_file(str(path).encode(), nx, ny, out.ctypes.data_as(_lib._c_float_p)))
    return out


def read_sources(path):
    """(srcpos [nsrc][8] in the reference's srcpos[1..8] order, TS)"""
    n = ctypes.c_int()
    sp = _lib._c_float_p()
    ts = ctypes.c_float()
    check(lib.dn_read_sources(str(path).encode(), ctypes.byref(n), ctypes.byref(sp), ctypes.byref(ts)))
    out = np.ctypeslib.as_array(sp, shape=(n.value, 8)).copy()
    _libc_free(sp)
    return out, ts.value


def read_signal_file(path):
    """rd_sour: the samples of a QUELLART 3 wavelet file (one per line)."""
    n = ctypes.c_int()
    sp = _lib._c_float_p()
    check(lib.dn_read_signal_file(str(path).encode(), ctypes.byref(n), ctypes.byref(sp)))
    out = np.ctypeslib.as_array(sp, shape=(max(n.value, 1),)).copy()[:n.value]
    _libc_free(sp)
    return out


def source_cell(x, y, dh):
    i, j = ctypes.c_int(), ctypes.c_int()
    check(lib.dn_source_cell(ctypes.c_float(x), ctypes.c_float(y), ctypes.c_float(dh), ctypes.byref(i),
                             ctypes.byref(j)))
    return i.value, j.value


def read_receivers(path, refrec, dh):
    ntr = ctypes.c_int()
    ri, rj = _lib._c_int_p(), _lib._c_int_p()
    rr = np.asarray(refrec, np.float32)
    check(lib.dn_read_receivers(str(path).encode(), rr.ctypes.data_as(_lib._c_float_p), ctypes.c_float(dh),
                                ctypes.byref(ntr), ctypes.byref(ri), ctypes.byref(rj)))
    a = np.ctypeslib.as_array(ri, shape=(ntr.value,)).copy() if ntr.value else np.zeros(0, np.int32)
    b = np.ctypeslib.as_array(rj, shape=(ntr.value,)).copy() if ntr.value else np.zeros(0, np.int32)
    _libc_free(ri)
    _libc_free(rj)
    return a, b


def write_su(path, section, ndt, dt, time, dh, rec_i, rec_j, refrec, xs, ys):
    sec = np.ascontiguousarray(section, np.float32)
    ri = np.ascontiguousarray(rec_i, np.int32)
    rj = np.ascontiguousarray(rec_j, np.int32)
    rr = np.asarray(refrec, np.float32)
    check(lib.dn_write_su(str(path).encode(), sec.ctypes.data_as(_lib._c_float_p), sec.shape[0], sec.shape[1], ndt,
                          ctypes.c_float(dt), ctypes.c_float(time), ctypes.c_float(dh),
                          ri.ctypes.data_as(_lib._c_int_p), rj.ctypes.data_as(_lib._c_int_p),
                          rr.ctypes.data_as(_lib._c_float_p), ctypes.c_float(xs), ctypes.c_float(ys)))


def write_seis(path, fmt, section, ndt, dt, time, dh, rec_i, rec_j, refrec, xs, ys):
    """dn_write_seis: SEIS_FORMAT fmt 1 (SU), 2 (ASCII) or 3 (binary float32)."""
    sec = np.ascontiguousarray(section, np.float32)
    ri = np.ascontiguousarray(rec_i, np.int32)
    rj = np.ascontiguousarray(rec_j, np.int32)
    rr = np.asarray(refrec, np.float32)
    check(lib.dn_write_seis(str(path).encode(), int(fmt), sec.ctypes.data_as(_lib._c_float_p), sec.shape[0],
                            sec.shape[1], ndt, ctypes.c_float(dt), ctypes.c_float(time), ctypes.c_float(dh),
                            ri.ctypes.data_as(_lib._c_int_p), rj.ctypes.data_as(_lib._c_int_p),
                            rr.ctypes.data_as(_lib._c_float_p), ctypes.c_float(xs), ctypes.c_float(ys)))


def read_su(path, ntr, ns):
    out = np.empty((ntr, ns), np.float32)
    check(lib.dn_read_su(str(path).encode(), ntr, ns, out.ctypes.data_as(_lib._c_float_p)))
    return out


def forward_inp(path, device=0):
    """MODE 0 of a parameter file on the GPU (SU files written where the file says)."""
    check(lib.dn_forward_inp(str(path).encode(), device))


_libc = ctypes.CDLL(None)
_libc.free.argtypes = [ctypes.c_void_p]


def _libc_free(p):
    _libc.free(ctypes.cast(p, ctypes.c_void_p))
