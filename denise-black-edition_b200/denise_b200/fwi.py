"""FWI outer loop: L-BFGS direction (FP64, on the device), the parabolic
step-length search of step_length_est_psv.c with calc_opt_step.c, and the
bounded model update of calc_mat_change_test_PSV.c.

One iteration (FWI_PSV.c): gradient and misfit of the current model over all
shots (batched, or sharded over ranks), search direction r = H g from the
L-BFGS history, test models x - eps r for a bracketing sequence of eps whose
misfits (forward runs, mode 2) fix a parabola, the model moved by its minimum.

The reference applies L-BFGS to its gradients after its normalisation steps
(store_LBFGS_PSV.c); here the model vector is [vp; vs; rho] divided per class
by the class maximum of the starting model, so the three classes are of the
same order, and the direction is scaled back before the update.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, lib


def calc_opt_step(L2t, epst):
    """Step length at the extremum of the parabola through (epst[k], L2t[k]) (FP64 solve)."""
    L = (ctypes.c_double * 3)(*[float(x) for x in L2t])
    e = (ctypes.c_float * 3)(*[float(x) for x in epst])
    out = ctypes.c_float()
    check(lib.dn_calc_opt_step(L, e, ctypes.byref(out)))
    return out.value


def mat_update(vp, vs, rho, dvp, dvs, drho, eps_scale, limits, iteration=1, inv_iter=(1, 1, 1), scalerho=1.0):
    """calc_mat_change_test_PSV: returns (vp, vs, rho, (EPSILON, EPSILON_u, EPSILON_rho))."""
    arrs = [np.ascontiguousarray(a, np.float32) for a in (vp, vs, rho, dvp, dvs, drho)]
    nx, ny = arrs[0].shape
    outs = [np.empty((nx, ny), np.float32) for _ in range(3)]
    lim = np.asarray(limits, np.float32)
    inv = np.asarray(inv_iter, np.int32)
    eps = np.zeros(3, np.float32)
    fp = _lib._c_float_p
    check(lib.dn_mat_update(nx, ny, *[a.ctypes.data_as(fp) for a in arrs], ctypes.c_float(eps_scale),
                            lim.ctypes.data_as(fp), int(iteration), inv.ctypes.data_as(_lib._c_int_p),
                            ctypes.c_float(scalerho), *[o.ctypes.data_as(fp) for o in outs], eps.ctypes.data_as(fp)))
    return outs[0], outs[1], outs[2], tuple(float(x) for x in eps)


def step_length(objective, L2_0, eps_scale=0.01, scalefac=2.0, stepmax=4):
    """step_length_est_psv.c: find eps_2 with L2(eps_2) < L2(0), then eps_3 beyond it
    with L2(eps_3) > L2(eps_2) (or give up after stepmax tries), and return the
    parabola's minimum.  objective(eps) -> misfit of the test model.  Returns
    (eps, L2t, epst, found) with 0-based arrays (index 0 = the current model)."""
    L2t = [float(L2_0), 0.0, 0.0]
    epst = [0.0, 0.0, 0.0]
    step1 = step2 = 0
    countstep = 0
    itests = iteste = 1
    found = True
    while step2 != 1 or step1 != 1:
        for itest in range(itests, iteste + 1):
            L2t[itest] = float(objective(eps_scale))
            epst[itest] = eps_scale
            epst[0] = 0.0
        if step1 == 0 and L2t[0] <= L2t[1]:
            eps_scale = eps_scale / scalefac
            countstep += 1
        if step1 == 1 and L2t[1] < L2t[2]:
            epst[2] = eps_scale
            step2 = 1
        if step1 == 1 and L2t[1] >= L2t[2]:
            epst[2] = eps_scale
            eps_scale = eps_scale + eps_scale / scalefac
            countstep += 1
        if step1 == 0 and L2t[0] > L2t[1]:
            epst[1] = eps_scale
            step1 = 1
            iteste = itests = 2
            countstep = 0
            eps_scale = eps_scale + eps_scale / scalefac
        if step1 == 0 and countstep > stepmax:
            found = False      # "Steplength estimation failed!"
            break
        if step1 == 1 and countstep > stepmax:
            step2 = 1          # no third step bracketing the minimum
    if step1 == 1:
        eps_scale = calc_opt_step(L2t, epst)
    return eps_scale, L2t, epst, found


class LBFGS:
    """Device-resident FP64 L-BFGS history (dn_lbfgs_*) over vectors of length n."""

    def __init__(self, n, m=20, device=0):
        import torch

        self.torch = torch
        self.dev = torch.device(f"cuda:{device}")
        self.n = n
        self.h = ctypes.c_void_p()
        check(lib.dn_lbfgs_create(int(n), int(m), int(device), ctypes.byref(self.h)))

    def _dev(self, x):
        t = self.torch
        return t.as_tensor(np.ascontiguousarray(x, np.float64)).to(self.dev) if isinstance(x, np.ndarray) else \
            x.to(self.dev, t.float64).contiguous()

    def push(self, s, y):
        ds, dy = self._dev(s), self._dev(y)
        self.torch.cuda.synchronize(self.dev)
        check(lib.dn_lbfgs_push(self.h, ds.data_ptr(), dy.data_ptr()))

    def count(self):
        c = ctypes.c_int()
        check(lib.dn_lbfgs_count(self.h, ctypes.byref(c)))
        return c.value

    def direction(self, g):
        dg = self._dev(g)
        dr = self.torch.empty_like(dg)
        self.torch.cuda.synchronize(self.dev)
        check(lib.dn_lbfgs_direction(self.h, dg.data_ptr(), dr.data_ptr()))
        return dr.cpu().numpy()

    def close(self):
        if self.h:
            lib.dn_lbfgs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def dot(a, b):
    """Deterministic FP64 dot product of two CUDA float64 tensors."""
    out = ctypes.c_double()
    check(lib.dn_dot(a.data_ptr(), b.data_ptr(), int(a.numel()), ctypes.byref(out)))
    return out.value


class FWI:
    """FWI iterations for one grid: shots (src_i, src_j, signals, rec_i, rec_j)
    with observed data obs[k] = (vx, vy) [ntr][nt]; `params` must store
    snapshots.  limits: (vp_lo, vp_hi, vs_lo, vs_hi, rho_lo, rho_hi).
    precond: a precond.PrecondConfig applied to every stacked gradient;
    shot_taper: (srtshape, srtradius, filtsize) of the per-shot circular taper;
    time_filter: (order, fc, fc_start) band-limiting sources and data;
    residual: calc_res options (Shot.residual_ex keywords) for gradient and
    misfit; energy: (C_vp, C_vs, C_rho) of the EPRECOND 1/3 scaling (params.eprecond
    set); inv_iter: (INV_VP_ITER, INV_VS_ITER, INV_RHO_ITER); test_shots: indices of
    the shots whose misfit is the objective and whose forward runs test the step
    lengths (TESTSHOT_START..END by INCR, grad_obj_psv.c and step_length_est_psv.c;
    None: all shots).  Shot tuples are (src_i, src_j, signals, rec_i, rec_j) with
    optional src_type, src_azi and the (x, z) source position in metres."""

    def __init__(self, params, model, shots, obs, limits, device=0, nlbfgs=20, eps_scale=0.01, scalefac=2.0,
                 stepmax=4, dist=None, precond=None, shot_taper=None, time_filter=None, residual=None, energy=None,
                 inv_iter=(1, 1, 1), test_shots=None):
        self.p = params
        self.vp, self.vs, self.rho = [np.ascontiguousarray(a, np.float32) for a in model[:3]]
        if time_filter is not None:
            # TIME_FILT (grad_obj_psv.c:151-155, calc_res_PSV.c): the source signals and the
            # observed data are band-limited by apply_tdfilt(ORDER, FC, FC_START)
            from .api import tdfilt

            order, fc, fc_start = time_filter
            shots = [tuple(sh[:2]) + (tdfilt(sh[2], params.dt, order, fc, fc_start, device),) + tuple(sh[3:])
                     for sh in shots]
            obs = [tuple(tdfilt(o, params.dt, order, fc, fc_start, device) for o in ob) for ob in obs]
        self.shots, self.obs, self.limits = shots, obs, limits
        self.residual, self.energy, self.inv_iter = residual, energy, tuple(inv_iter)
        self.test_shots = None if test_shots is None else sorted(set(int(k) for k in test_shots))
        self.device, self.dist = device, dist
        self.eps_scale, self.scalefac, self.stepmax = eps_scale, scalefac, stepmax
        self.scale = np.array([self.vp.max(), self.vs.max(), self.rho.max()], np.float64)
        n = 3 * params.nx * params.ny
        self.lbfgs = LBFGS(n, nlbfgs, device)
        # gradient conditioning after stacking (FWI_PSV.c:628-634) and per shot
        self.shot_taper = shot_taper
        self.precond = None
        if precond is not None:
            from .precond import PrecondPlan

            self.precond = PrecondPlan(params.nx, params.ny, params.dh, precond, device)
        self.prev = None          # (x, g) of the previous iteration, scaled
        self.history = []

    def _x(self):
        return np.concatenate([(a.astype(np.float64) / s).ravel() for a, s in zip((self.vp, self.vs, self.rho),
                                                                                   self.scale)])

    def gradient(self, model=None):
        from .shard import sharded_gradient

        m = model or (self.vp, self.vs, self.rho)
        g_vp, g_vs, g_rho, L2 = sharded_gradient(self.p, m, self.shots, self.obs, self.dist, self.device,
                                                 self.shot_taper, self.residual, self.energy, self.test_shots)
        if self.precond is not None:
            from . import api as dn

            dm = dn.Model(self.p.replace(store_snapshots=0, ckpt_steps=0, L=0, fl=()), *m[:3], device=self.device)
            dm.set_gradient(g_vp.astype(np.float32), g_vs.astype(np.float32), g_rho.astype(np.float32))
            self.precond.apply(dm)
            g_vp, g_vs, g_rho = [x.astype(np.float64) for x in dm.gradient()]
            dm.close()
        return g_vp, g_vs, g_rho, L2

    def misfit(self, model):
        """mode-2 forward runs of all shots on a test model; sum of the vx and vy misfits."""
        from . import api as dn

        from .shard import make_shot, source_position

        from .shard import memory_batches

        p = self.p.replace(store_snapshots=0, ckpt_steps=0)
        m = dn.Model(p, *model, device=self.device)
        idx = range(len(self.shots)) if self.test_shots is None else self.test_shots
        L2 = 0.0
        for part in memory_batches(p, self.shots, idx, 0, self.device):
            ss = [make_shot(m, self.shots[k]) for k in part]
            dn.run(ss, _lib.MODE_OBJECTIVE)
            for s, k in zip(ss, part):
                sh, (ovx, ovy) = self.shots[k], self.obs[k]
                if self.residual is None:
                    L2 += s.residual(ovx, _lib.SEC_VX) + s.residual(ovy, _lib.SEC_VY)
                else:
                    sx, sz = source_position(sh, self.p.dh)
                    opts = dict({"src_x": sx, "src_z": sz}, **self.residual)
                    L2 += s.residual_ex(ovx, _lib.SEC_VX, **opts) + s.residual_ex(ovy, _lib.SEC_VY, **opts)
            for s in ss:
                s.close()
        m.close()
        return L2

    def iterate(self, it):
        import time

        t0 = time.perf_counter()
        g_vp, g_vs, g_rho, L2 = self.gradient()
        t1 = time.perf_counter()
        nx, ny = self.p.nx, self.p.ny
        # gradient with respect to the scaled model x = m / scale
        g = np.concatenate([(gc * s).ravel() for gc, s in zip((g_vp, g_vs, g_rho), self.scale)])
        x = self._x()
        if self.prev is not None:
            self.lbfgs.push(x - self.prev[0], g - self.prev[1])
        self.prev = (x, g)
        r = self.lbfgs.direction(g)
        d = [(r[k * nx * ny:(k + 1) * nx * ny] / self.scale[k]).reshape(nx, ny).astype(np.float32) for k in range(3)]
        t2 = time.perf_counter()
        ntests = [0]

        def objective(eps):
            ntests[0] += 1
            vp, vs, rho, _ = mat_update(self.vp, self.vs, self.rho, *d, eps, self.limits, it, self.inv_iter)
            return self.misfit((vp, vs, rho))

        eps, L2t, epst, found = step_length(objective, L2, self.eps_scale, self.scalefac, self.stepmax)
        if found:
            self.vp, self.vs, self.rho, _ = mat_update(self.vp, self.vs, self.rho, *d, eps, self.limits, it,
                                                       self.inv_iter)
        t3 = time.perf_counter()
        self.history.append({"iteration": it, "misfit": L2, "eps": eps, "L2t": L2t, "epst": epst, "found": found,
                             "gradient_s": t1 - t0, "lbfgs_s": t2 - t1, "step_search_s": t3 - t2,
                             "test_models": ntests[0]})
        return L2


def rtm_image(params, model, shots, obs, device=0, batch=None):
    """Reverse-time migration (RTM_PSV.c): per shot, a forward run with
    snapshots, the observed data as adjoint source (dn_shot_rtm_source) and the
    adjoint run; the images are the stacked vp and vs gradients (the P and S
    images RTM_PSV_out.c writes).  `params` must store snapshots.  Returns
    (P image, S image) in file order."""
    from . import api as dn
    from .shard import make_shot

    m = dn.Model(params, *model[:3], model[3] if params.L else None, model[4] if params.L else None,
                 device=device)
    batch = batch or len(shots)
    for b0 in range(0, len(shots), batch):
        ss = [make_shot(m, sh) for sh in shots[b0:b0 + batch]]
        dn.run(ss, _lib.MODE_FORWARD)
        for s, (ovx, ovy) in zip(ss, obs[b0:b0 + batch]):
            s.rtm_source(ovx, _lib.SEC_VX)
            s.rtm_source(ovy, _lib.SEC_VY)
        dn.run(ss, _lib.MODE_ADJOINT)
        for s in ss:
            s.accumulate_gradient()
            s.close()
    g = m.gradient()
    m.close()
    return g[0], g[1]
