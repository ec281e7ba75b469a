"""Gradient conditioning: smooth_grad (src/smooth_grad.c) and precond_PSV
(src/PSV/precond_PSV.c) on the device, through dn_precond_create/apply.

    cfg = PrecondConfig(spatfilter=4, wd_damp=0.5, wd_damp1=0.5, fc_end=10.0,
                        taper_hor=1, gradt=(5, 12, 0, 12), exp_taper_grad_hor=2.0)
    plan = PrecondPlan(nx, ny, dh, cfg)
    plan.apply(model)            # the model's stacked gradients, in place
"""
import ctypes
from dataclasses import dataclass, field
from typing import Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import check, lib


@dataclass
class PrecondConfig:
    """The .inp switches of the gradient conditioning (names in lower case)."""
    spatfilter: int = 0                  # 0 none, 2 smooth2, 3 gauss_filt, 4 gauss_filt_var
    wd_damp: float = 0.0
    wd_damp1: float = 0.0
    fc_end: float = 0.0
    c_vs: float = 0.0                    # gauss_filt reference velocity
    taper_vert: int = 0                  # SWS_TAPER_GRAD_VERT
    taper_hor: int = 0                   # SWS_TAPER_GRAD_HOR
    taper_sources: int = 0               # SWS_TAPER_GRAD_SOURCES
    taper_file: int = 0                  # SWS_TAPER_FILE
    gradt: Tuple[int, int, int, int] = (0, 0, 0, 0)
    exp_taper_grad_hor: float = 0.0
    srtshape: int = 1
    srtradius: float = 0.0
    filtsize: int = 0
    taper_files: Optional[Sequence[np.ndarray]] = None    # vp, vs, rho coefficient arrays (nx, ny), file order
    sources: Sequence[Tuple[float, float]] = field(default_factory=list)   # (x, z) in metres
    receivers: Sequence[Tuple[int, int]] = field(default_factory=list)     # (i, j) grid indices

    def to_c(self):
        """The dn_precond structure and the arrays it points to (keep both alive)."""
        c = _lib.Precond()
        for k in ("spatfilter", "wd_damp", "wd_damp1", "fc_end", "c_vs", "taper_vert", "taper_hor", "taper_sources",
                  "taper_file", "exp_taper_grad_hor", "srtshape", "srtradius", "filtsize"):
            setattr(c, k, getattr(self, k))
        c.gradt[:] = [int(x) for x in self.gradt]
        keep = []
        if self.taper_files is not None:
            arrs = [np.ascontiguousarray(a, np.float32) for a in self.taper_files]
            keep += arrs
            c.taper_vp, c.taper_vs, c.taper_rho = (_lib.fptr(a) for a in arrs)
        sx = np.ascontiguousarray([s[0] for s in self.sources] or [0.0], np.float32)
        sz = np.ascontiguousarray([s[1] for s in self.sources] or [0.0], np.float32)
        ri = np.ascontiguousarray([r[0] for r in self.receivers] or [0], np.int32)
        rj = np.ascontiguousarray([r[1] for r in self.receivers] or [0], np.int32)
        keep += [sx, sz, ri, rj]
        c.nsrc, c.src_x, c.src_z = len(self.sources), _lib.fptr(sx), _lib.fptr(sz)
        c.ntr, c.rec_i, c.rec_j = len(self.receivers), _lib.iptr(ri), _lib.iptr(rj)
        return c, keep


class PrecondPlan:
    """dn_precond_plan for one grid: the geometry-dependent parts on the device."""

    def __init__(self, nx, ny, dh, cfg: PrecondConfig, device=0):
        self.nx, self.ny = nx, ny
        c, keep = cfg.to_c()
        h = ctypes.c_void_p()
        check(lib.dn_precond_create(int(nx), int(ny), ctypes.c_float(dh), ctypes.byref(c), int(device),
                                    ctypes.byref(h)))
        self.handle = h

    def apply(self, model):
        check(lib.dn_precond_apply(self.handle, model.handle))

    def close(self):
        if self.handle:
            lib.dn_precond_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def taper_coefficients(nx, ny, dh, cfg: PrecondConfig, sws):
    """taper_grad's coefficients of switch sws (1 vertical, 2 horizontal, 3 sources), file order (nx, ny)."""
    c, keep = cfg.to_c()
    out = np.zeros((nx, ny), np.float32)
    check(lib.dn_taper_coefficients(int(nx), int(ny), ctypes.c_float(dh), ctypes.byref(c), int(sws),
                                    _lib.fptr(out)))
    return out
