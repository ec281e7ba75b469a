"""Test-side access to the CPU oracles (never imported by the product).

* ``Restatement`` - oracle/liboracle_psv.so, this project's C restatement of
  the reference scheme in float (bit-identical to the reference) and double.
* ``Reference``   - oracle/_ref/libdenise_ref.so, the reference's own sources
  built by oracle/Makefile, driven through oracle/ref_harness.c.  Present
  where it was built (it is git-ignored); tests that need it skip otherwise.
"""
import ctypes
import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle")
REST_SO = os.path.join(ORACLE, "liboracle_psv.so")
REF_SO = os.path.join(ORACLE, "_ref", "libdenise_ref.so")
REF_BIN = os.path.join(ORACLE, "_ref", "denise")

_f = ctypes.POINTER(ctypes.c_float)
_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)


def _fp(a):
    return None if a is None else np.ascontiguousarray(a, np.float32).ctypes.data_as(_f)


def _ip(a):
    return None if a is None else np.ascontiguousarray(a, np.int32).ctypes.data_as(_i)


def params_arrays(p, honor_q=0):
    ip = np.array([p.nx, p.ny, p.nt, p.fdorder, p.maxrelerror, p.free_surf, p.fw, p.L, p.quelltypb,
                   max(p.dtinv, 1), p.seismo, p.eprecond, honor_q, 0, 0, 0], np.int32)
    fl = list(p.fl) + [0.0] * (5 - len(p.fl))
    fp = np.array([p.dh, p.dt, p.damping, p.fpml, p.npower, p.k_max_pml, p.ts] + fl, np.float32)
    return ip, fp


def build_restatement():
    if not os.path.exists(REST_SO):
        subprocess.check_call(["make", "-s", "-C", ORACLE, "restatement"])
    return REST_SO


class Restatement:
    """One shot of the CPU restatement; precision 'f' (float) or 'd' (double)."""

    def __init__(self, p, model, src, rec, prec="f", honor_q=0):
        self.lib = ctypes.CDLL(build_restatement())
        self.p, self.prec = p, prec
        self.real = np.float32 if prec == "f" else np.float64
        sfx = "_" + prec
        self.fn = {n: getattr(self.lib, "or_" + n + sfx) for n in
                   ("create", "destroy", "forward", "adjoint", "get_sections", "get_field", "get_gradient",
                    "get_setup")}
        self.fn["create"].restype = ctypes.c_void_p
        for n in ("destroy", "forward", "adjoint", "get_sections", "get_field", "get_gradient", "get_setup"):
            self.fn[n].argtypes = None
        vp, vs, rho = model[:3]
        qp, qs = (model[3], model[4]) if len(model) > 3 else (None, None)
        si, sj, sig = src[:3]
        styp = src[3] if len(src) > 3 else None
        sazi = src[4] if len(src) > 4 else None
        ri, rj = rec
        ip, fp = params_arrays(p, honor_q)
        self._keep = [np.ascontiguousarray(a, np.float32) if a is not None else None
                      for a in (vp, vs, rho, qp, qs, sig, sazi)]
        self.ntr = len(ri)
        self.h = ctypes.c_void_p(self.fn["create"](
            _ip(ip), _fp(fp), *[_fp(a) for a in self._keep[:5]], ctypes.c_int(len(si)), _ip(si), _ip(sj),
            _ip(styp), _fp(self._keep[6]), _fp(self._keep[5]), ctypes.c_int(len(ri)), _ip(ri), _ip(rj)))

    def _out(self, shape):
        a = np.zeros(shape, self.real)
        return a, a.ctypes.data_as(_f if self.prec == "f" else _d)

    def forward(self, store=False, nt_stop=0):
        st = self.fn["forward"](self.h, ctypes.c_int(int(store)), ctypes.c_int(nt_stop))
        assert st == 0, st

    def adjoint(self, res_vx=None, res_vy=None, res_p=None):
        st = self.fn["adjoint"](self.h, _fp(res_vx), _fp(res_vy), _fp(res_p))
        assert st == 0, st

    def sections(self, comp=0):
        a, ptr = self._out((self.ntr, self.p.nt))
        self.fn["get_sections"](self.h, ctypes.c_int(comp), ptr)
        return a

    def field(self, fid):
        a, ptr = self._out((self.p.nx, self.p.ny))
        self.fn["get_field"](self.h, ctypes.c_int(fid), ptr)
        return a

    def gradient(self):
        outs = [self._out((self.p.nx, self.p.ny)) for _ in range(3)]
        self.fn["get_gradient"](self.h, *[o[1] for o in outs])
        return tuple(o[0] for o in outs)

    def setup(self, which):
        shape = 7 if which == 0 else (20 * 2 * self.p.fw if which == 1 else (self.p.nx, self.p.ny))
        a, ptr = self._out(shape)
        self.fn["get_setup"](self.h, ctypes.c_int(which), ptr)
        return a

    def __del__(self):
        try:
            self.fn["destroy"](self.h)
        except Exception:
            pass


def reference_available():
    return os.path.exists(REF_SO)


def write_model_files(prefix, vp, vs, rho, qp=None, qs=None):
    """Binary float32 model files in the reference's x-major order (readmod_elastic_PSV.c:72-85)."""
    for ext, a in (("vp", vp), ("vs", vs), ("rho", rho), ("qp", qp), ("qs", qs)):
        if a is not None:
            np.ascontiguousarray(a, np.float32).tofile(f"{prefix}.{ext}")


class Reference:
    """One shot of the reference's own code (single-rank harness).  The harness
    keeps global state, so run each case in a fresh process (see run_isolated)."""

    def __init__(self, p, model, src, rec, mode_global=1, workdir=None):
        self.lib = ctypes.CDLL(REF_SO)
        self.lib.refh_calc_res.restype = ctypes.c_double
        self.p = p
        self.workdir = workdir or tempfile.mkdtemp(prefix="dnref_")
        prefix = os.path.join(self.workdir, "model")
        vp, vs, rho = model[:3]
        qp = model[3] if len(model) > 3 else np.full_like(vp, 30.0)
        qs = model[4] if len(model) > 4 else np.full_like(vp, 30.0)
        write_model_files(prefix, vp, vs, rho, qp, qs)
        ip = np.array([p.nx, p.ny, p.nt, p.fdorder, p.maxrelerror, p.free_surf, p.fw, p.L, p.quelltypb,
                       max(p.dtinv, 1), p.seismo, p.eprecond, mode_global], np.int32)
        fl = list(p.fl) + [0.0] * (5 - len(p.fl))
        fp = np.array([p.dh, p.dt, p.damping, p.fpml, p.npower, p.k_max_pml, p.ts] + fl, np.float32)
        assert self.lib.refh_setup(_ip(ip), _fp(fp), prefix.encode()) == 0
        si, sj, sig = src[:3]
        styp = src[3] if len(src) > 3 else np.ones(len(si))
        sazi = src[4] if len(src) > 4 else np.zeros(len(si))
        ns = len(si)
        srcpos = np.zeros((8, ns), np.float32)
        srcpos[0], srcpos[1], srcpos[6], srcpos[7] = si, sj, sazi, styp
        self.ntr = len(rec[0])
        self._keep = (srcpos, np.ascontiguousarray(sig, np.float32))
        assert self.lib.refh_set_acq(ctypes.c_int(ns), _fp(srcpos), _fp(self._keep[1]), ctypes.c_int(self.ntr),
                                     _ip(rec[0]), _ip(rec[1])) == 0

    def __del__(self):
        import shutil

        shutil.rmtree(self.workdir, ignore_errors=True)

    def hc(self):
        a = np.zeros(7, np.float32)
        self.lib.refh_get_hc(_fp(a))
        return a

    def pml(self):
        a = np.zeros(20 * 2 * self.p.fw, np.float32)
        self.lib.refh_get_pml(a.ctypes.data_as(_f))
        return a

    def mat(self, which):
        a = np.zeros((self.p.nx, self.p.ny), np.float32)
        assert self.lib.refh_get_mat(ctypes.c_int(which), a.ctypes.data_as(_f)) == 0
        return a

    def visc_vectors(self):
        a = np.zeros(5 * self.p.L, np.float32)
        self.lib.refh_get_visc_vectors(a.ctypes.data_as(_f))
        return a.reshape(5, self.p.L)

    def run(self, mode):
        self.lib.refh_run(ctypes.c_int(mode))

    def sections(self, comp=0):
        a = np.zeros((self.ntr, self.p.nt), np.float32)
        assert self.lib.refh_get_sections(ctypes.c_int(comp), a.ctypes.data_as(_f)) == 0
        return a

    def set_residuals(self, vx=None, vy=None, p=None):
        self._res = [np.ascontiguousarray(x, np.float32) if x is not None else None for x in (vx, vy, p)]
        self.lib.refh_set_residuals(*[_fp(x) for x in self._res])

    def calc_res(self, data, syn):
        diff = np.zeros((self.ntr, self.p.nt), np.float32)
        l2 = self.lib.refh_calc_res(_fp(data), _fp(syn), diff.ctypes.data_as(_f))
        return diff, l2

    def field(self, fid):
        a = np.zeros((self.p.nx, self.p.ny), np.float32)
        assert self.lib.refh_get_field(ctypes.c_int(fid), a.ctypes.data_as(_f)) == 0
        return a

    def snapshot(self, k, f):
        a = np.zeros((self.p.nx, self.p.ny), np.float32)
        self.lib.refh_get_snapshot(ctypes.c_int(k), ctypes.c_int(f), a.ctypes.data_as(_f))
        return a

    def ass_grad(self):
        g = [np.zeros((self.p.nx, self.p.ny), np.float32) for _ in range(3)]
        self.lib.refh_ass_grad(*[x.ctypes.data_as(_f) for x in g])
        return tuple(g)

    def ass_grad_ep(self, c_vp, c_vs, c_rho):
        """ass_gradPSV + the per-shot energy preconditioning (EPRECOND of the set-up)."""
        g = [np.zeros((self.p.nx, self.p.ny), np.float32) for _ in range(3)]
        c = np.array([c_vp, c_vs, c_rho], np.float32)
        self.lib.refh_ass_grad_ep(c.ctypes.data_as(_f), *[x.ctypes.data_as(_f) for x in g])
        return tuple(g)


def run_isolated(fn, *args, timeout=600):
    """Runs fn(*args) in a fresh spawned process (the reference keeps globals).
    A reference error exits that process (its err() calls exit); that surfaces
    here as BrokenProcessPool instead of a wait without end."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    with ProcessPoolExecutor(max_workers=1, mp_context=mp.get_context("spawn")) as ex:
        return ex.submit(fn, *args).result(timeout=timeout)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


def reference_forward_sections(p, model, src, rec):
    """vx and vy sections of one forward run of the reference's code (run it in a fresh process)."""
    r = Reference(p, model, src, rec, mode_global=0)
    r.run(0)
    return r.sections(0), r.sections(1)


# ---------------------------------------------------------------------------
# the reference's gradient conditioning (precond_PSV, taper_grad_shot,
# smooth_grad) through oracle/ref_harness.c; call each in run_isolated().
# Gradients are [NY][NX] float32 (row j, column i); the harness takes file order.
# ---------------------------------------------------------------------------
def _ref_lib():
    return ctypes.CDLL(REF_SO)


def ref_precond(workdir, nx, ny, dh, sw, gradt, exp_hor, srtshape, srtradius, filtsize, srcs, recs, grads,
                tfile="tp"):
    os.chdir(workdir)
    lib = _ref_lib()
    gs = [np.ascontiguousarray(np.asarray(g, np.float32).T) for g in grads]
    sxz = np.asarray(srcs, np.float32).reshape(-1, 2) if len(srcs) else np.zeros((1, 2), np.float32)
    ri = np.array([r[0] for r in recs] or [0], np.int32)
    rj = np.array([r[1] for r in recs] or [0], np.int32)
    lib.refh_precond(ctypes.c_int(nx), ctypes.c_int(ny), ctypes.c_float(dh), _ip(sw), _ip(gradt),
                     ctypes.c_float(exp_hor), ctypes.c_int(srtshape), ctypes.c_float(srtradius), ctypes.c_int(filtsize),
                     tfile.encode(), ctypes.c_int(len(srcs)), _fp(sxz), ctypes.c_int(len(recs)), _ip(ri), _ip(rj),
                     *[g.ctypes.data_as(_f) for g in gs])
    return [g.T.copy() for g in gs]


def ref_taper_shot(workdir, nx, ny, dh, srtshape, srtradius, filtsize, srcs, ishot, grad, tfile="tp"):
    os.chdir(workdir)
    lib = _ref_lib()
    g = np.ascontiguousarray(np.asarray(grad, np.float32).T)
    sxz = np.asarray(srcs, np.float32).reshape(-1, 2)
    lib.refh_taper_shot(ctypes.c_int(nx), ctypes.c_int(ny), ctypes.c_float(dh), ctypes.c_int(srtshape),
                        ctypes.c_float(srtradius), ctypes.c_int(filtsize), tfile.encode(), ctypes.c_int(len(srcs)),
                        _fp(sxz), ctypes.c_int(ishot), g.ctypes.data_as(_f))
    return g.T.copy()


def ref_smooth_grad(workdir, nx, ny, dh, spatfilter, wd_damp, wd_damp1, fc_end, c_vs, vel, grad, jac="jac"):
    os.chdir(workdir)
    lib = _ref_lib()
    g = np.ascontiguousarray(np.asarray(grad, np.float32).T)
    v = np.ascontiguousarray(np.asarray(vel, np.float32).T)
    lib.refh_smooth_grad(ctypes.c_int(nx), ctypes.c_int(ny), ctypes.c_float(dh), ctypes.c_int(spatfilter),
                         ctypes.c_float(wd_damp), ctypes.c_float(wd_damp1), ctypes.c_float(fc_end), ctypes.c_float(c_vs),
                         jac.encode(), v.ctypes.data_as(_f), g.ctypes.data_as(_f))
    return g.T.copy()


def ref_calc_res_ex(workdir, data, syn, dt, dh, iopt, fopt, rec_i, rec_j, src, kill=None):
    """The reference's calc_res with the options of refh_calc_res_ex; run it in run_isolated()."""
    os.chdir(workdir)
    lib = _ref_lib()
    lib.refh_calc_res_ex.restype = ctypes.c_double
    d = np.ascontiguousarray(data, np.float32)
    s = np.ascontiguousarray(syn, np.float32)
    ntr, ns = d.shape
    out = np.zeros_like(d)
    killfile = None
    if kill is not None:
        with open("kill.dat", "w") as f:
            f.write(" ".join(str(int(k)) for k in kill) + "\n")
        killfile = b"kill.dat"
    l2 = lib.refh_calc_res_ex(ctypes.c_int(ntr), ctypes.c_int(ns), ctypes.c_float(dt), ctypes.c_float(dh),
                              _ip(np.asarray(iopt, np.int32)), _fp(np.asarray(fopt, np.float32)), _ip(rec_i),
                              _ip(rec_j), ctypes.c_float(src[0]), ctypes.c_float(src[1]), killfile,
                              d.ctypes.data_as(_f), s.ctypes.data_as(_f), out.ctypes.data_as(_f))
    return out, l2


def ref_wavelet_ex(workdir, quellart, n_order, nt, dt, tshift, fc, amp, fc_spike_1=0.0, fc_spike_2=0.0, ts=0.0,
                   signal=None, ishot=1, filt_order=0):
    """The reference's wavelet() (and, for QUELLART 6 with filt_order > 0, the
    apply_tdfilt of FD_PSV.c:324-331) for one source; QUELLART 3 reads
    `signal` from "sig_shot_<ishot>.dat" in workdir.  Run it in run_isolated()."""
    os.chdir(workdir)
    lib = _ref_lib()
    if signal is not None:
        with open(f"sig_shot_{ishot}.dat", "w") as f:
            f.write("".join(f"{float(v):.9e}\n" for v in np.asarray(signal, np.float32)))
    out = np.zeros(nt, np.float32)
    lib.refh_wavelet_ex(ctypes.c_int(quellart), ctypes.c_int(n_order), ctypes.c_int(nt), ctypes.c_float(dt),
                        ctypes.c_float(tshift), ctypes.c_float(fc), ctypes.c_float(amp), ctypes.c_float(fc_spike_1),
                        ctypes.c_float(fc_spike_2), ctypes.c_float(ts), b"sig", ctypes.c_int(ishot),
                        ctypes.c_int(filt_order), out.ctypes.data_as(_f))
    return out


def ref_apply_tdfilt(data, dt, order, fc2, fc1):
    """The reference's apply_tdfilt on [ntr][ns] float32 traces; run it in run_isolated()."""
    lib = _ref_lib()
    d = np.ascontiguousarray(data, np.float32).copy()
    lib.refh_apply_tdfilt(ctypes.c_int(d.shape[0]), ctypes.c_int(d.shape[1]), ctypes.c_float(dt), ctypes.c_int(order),
                          ctypes.c_float(fc2), ctypes.c_float(fc1), d.ctypes.data_as(_f))
    return d
