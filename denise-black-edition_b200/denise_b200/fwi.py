"""FWI outer loop of FWI_PSV.c: the gradient on the device (sharded over
ranks), the reference's optimisers (L-BFGS of store_LBFGS_PSV.c / LBFGS.c /
extract_LBFGS_PSV.c and PCG of PCG.c on the device, float vectors with FP64
dot products), the parabolic step-length search of step_length_est_psv.c with
calc_opt_step.c, and the bounded model update of calc_mat_change_test_PSV.c.

One iteration: gradient and misfit of the current model over all shots,
conditioning, the search direction of the optimiser, test models m - eps d for
a bracketing sequence of eps whose misfits (forward runs, mode 2) fix a
parabola, the model moved by its minimum.

LBFGS (dn_lbfgs_*) is a general FP64 L-BFGS on device vectors; the FWI
iteration uses Optimizer, the reference's own scheme.
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
    f32 = np.float32
    eps_scale, scalefac = f32(eps_scale), f32(scalefac)     # float in step_length_est_psv.c
    L2t = [float(L2_0), 0.0, 0.0]
    epst = [f32(0.0), f32(0.0), f32(0.0)]
    step1 = step2 = 0
    countstep = 0
    itests = iteste = 1
    found = True
    while step2 != 1 or step1 != 1:
        for itest in range(itests, iteste + 1):
            L2t[itest] = float(objective(float(eps_scale)))
            epst[itest] = eps_scale
            epst[0] = f32(0.0)
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
        eps_scale = f32(calc_opt_step(L2t, epst))
    return float(eps_scale), L2t, [float(x) for x in epst], found


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


class Optimizer:
    """The reference's optimiser on the device (dn_optim_*): GRAD_METHOD 2,
    L-BFGS with NLBFGS pairs, or 1, PCG with PCG_BETA (FWI_PSV.c:637-676).
    step() replaces a Model's stacked gradient by the search direction; the
    history persists across iterations and stages until reset() (FWI_PSV.c
    zeroes it only when a stage ends by its abort criterion)."""

    FILES = ("p", "p_u", "p_rho", "p_vp", "p_vs", "p_mrho", "c", "c_u", "c_rho")

    def __init__(self, grad_method, nx, ny, nlbfgs=20, pcg_beta=2, device=0):
        self.grad_method, self.nx, self.ny, self.device = int(grad_method), nx, ny, device
        self.h = None
        if self.grad_method in (1, 2):
            self.h = ctypes.c_void_p()
            check(lib.dn_optim_create(self.grad_method, int(nx), int(ny), int(nlbfgs), int(pcg_beta), int(device),
                                      ctypes.byref(self.h)))

    def step(self, model, it, c):
        """Any other GRAD_METHOD leaves the conditioned gradient as the direction, as FWI_PSV.c does."""
        if self.h is None:
            return
        cc = (ctypes.c_float * 3)(*[float(x) for x in c])
        check(lib.dn_optim_step(self.h, model.handle, int(it), cc))

    def reset(self):
        if self.h is not None:
            check(lib.dn_optim_reset(self.h))

    def vector(self, which):
        """The JACOBIAN vector `which` (0-8, FILES order) after an L-BFGS step, [nx][ny] float32."""
        out = np.empty((self.nx, self.ny), np.float32)
        check(lib.dn_optim_get(self.h, int(which), _lib.fptr(out)))
        return out

    def write_jacobian(self, prefix):
        """The files extract_LBFGS_PSV.c:80-248 writes after an L-BFGS step:
        <JACOBIAN>_{p,p_u,p_rho}.old (normalised gradients), _{p_vp,p_vs,p_mrho}.old
        (the model), _{c,c_u,c_rho}.old (the direction), each also as the one-rank
        part file <name>.0.0 that mergemod merges (identical on one rank)."""
        if self.grad_method != 2:
            return
        for k, name in enumerate(self.FILES):
            a = self.vector(k)
            for path in (f"{prefix}_{name}.old.0.0", f"{prefix}_{name}.old"):
                a.tofile(path)

    def close(self):
        if self.h:
            lib.dn_optim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_inv_model(prefix, model):
    """The files calc_mat_change_test_PSV.c:223-243 writes with every model
    update: <INV_MODELFILE>_{vp,vs,rho}.bin and their one-rank part files .0.0."""
    for name, a in zip(("vp", "vs", "rho"), model):
        a = np.ascontiguousarray(a, np.float32)
        for path in (f"{prefix}_{name}.bin.0.0", f"{prefix}_{name}.bin"):
            a.tofile(path)


class FWI:
    """FWI iterations of FWI_PSV.c for one grid: shots (src_i, src_j, signals,
    rec_i, rec_j) with observed data obs[k] = (vx, vy) [ntr][nt]; `params` must
    store snapshots.  limits: (vp_lo, vp_hi, vs_lo, vs_hi, rho_lo, rho_hi).

    One iteration: the gradient of all shots (batched, sharded over the ranks of
    `dist`, summed on the device), its conditioning (precond: smooth_grad and
    precond_PSV), the reference's optimiser (grad_method 2 L-BFGS with nlbfgs
    pairs, 1 PCG with pcg_beta; the gradients normalised by `averages` = C_vp,
    C_vs, C_rho, the starting model's averages), the parabolic step search of
    step_length_est_psv.c with mode-2 forward runs of the test shots (sharded
    the same way), and the bounded update of calc_mat_change_test_PSV.c.

    precond: a precond.PrecondConfig; shot_taper: (srtshape, srtradius,
    filtsize) of the per-shot circular taper; time_filter: (order, fc,
    fc_start) band-limiting sources and data; residual: calc_res options
    (Shot.residual_ex keywords) for gradient and misfit; energy: (C_vp, C_vs,
    C_rho) of the EPRECOND 1/3 scaling (params.eprecond set); inv_iter:
    (INV_VP_ITER, INV_VS_ITER, INV_RHO_ITER); scalerho: SCALERHO; test_shots:
    indices of the shots whose misfit is the objective and whose forward runs
    test the step lengths (TESTSHOT_START..END by INCR; None: all shots);
    optimizer: an Optimizer to continue (the workflow keeps one across stages)
    or None for a new one; jacobian: the JACOBIAN prefix of the files
    extract_LBFGS_PSV writes (None: none); inv_modelfile: the INV_MODELFILE
    prefix of the files every update writes (None: none).  Shot tuples are
    (src_i, src_j, signals, rec_i, rec_j) with optional src_type, src_azi and
    the (x, z) source position in metres."""

    def __init__(self, params, model, shots, obs, limits, device=0, nlbfgs=20, eps_scale=0.01, scalefac=2.0,
                 stepmax=4, dist=None, precond=None, shot_taper=None, time_filter=None, residual=None, energy=None,
                 inv_iter=(1, 1, 1), test_shots=None, grad_method=2, pcg_beta=2, averages=None, optimizer=None,
                 jacobian=None, inv_modelfile=None, scalerho=1.0):
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
        self.residual, self.energy, self.inv_iter, self.scalerho = residual, energy, tuple(inv_iter), scalerho
        self.test_shots = None if test_shots is None else sorted(set(int(k) for k in test_shots))
        self.device, self.dist = device, dist
        self.eps_scale, self.scalefac, self.stepmax = eps_scale, scalefac, stepmax
        if averages is None:
            from .workflow import model_averages

            averages = model_averages(self.vp, self.vs, self.rho)
        self.averages = tuple(float(x) for x in averages)
        self.own_optimizer = optimizer is None
        self.optimizer = optimizer or Optimizer(grad_method, params.nx, params.ny, nlbfgs, pcg_beta, device)
        self.jacobian, self.inv_modelfile = jacobian, inv_modelfile
        self.rank0 = dist is None or not dist.is_initialized() or dist.get_rank() == 0
        # gradient conditioning after stacking (FWI_PSV.c:628-634) and per shot
        self.shot_taper = shot_taper
        self.precond = None
        if precond is not None:
            from .precond import PrecondPlan

            self.precond = PrecondPlan(params.nx, params.ny, params.dh, precond, device)
        self.history = []

    def _gradient_model(self, model=None):
        from .shard import gradient_model

        m = model or (self.vp, self.vs, self.rho)
        gm, L2 = gradient_model(self.p, m, self.shots, self.obs, self.dist, self.device, self.shot_taper,
                                self.residual, self.energy, self.test_shots)
        if self.precond is not None:
            self.precond.apply(gm)
        return gm, L2

    def gradient(self, model=None):
        """The stacked, conditioned gradient and the misfit: (g_vp, g_vs, g_rho, L2) on the host."""
        gm, L2 = self._gradient_model(model)
        try:
            g = [x.astype(np.float64) for x in gm.gradient()]
        finally:
            gm.close()
        return g[0], g[1], g[2], L2

    def misfit(self, model):
        """obj_psv: the misfit of the test shots on a test model (mode-2 forward runs, sharded)."""
        from .shard import sharded_misfit

        idx = range(len(self.shots)) if self.test_shots is None else self.test_shots
        return sharded_misfit(self.p, model, self.shots, self.obs, idx, self.dist, self.device, self.residual)

    def iterate(self, it, min_iter=0):
        """Iteration `it` (FWI_PSV.c's per-stage counter) of a stage with MIN_ITER
        min_iter.  Returns the misfit of the current model (L2t[4])."""
        import time

        t0 = time.perf_counter()
        gm, L2 = self._gradient_model()
        try:
            t1 = time.perf_counter()
            self.optimizer.step(gm, it, self.averages)
            if self.jacobian is not None and self.rank0:
                self.optimizer.write_jacobian(self.jacobian)
            d = gm.gradient()
        finally:
            gm.close()
        t2 = time.perf_counter()
        ntests = [0]

        def objective(eps):
            ntests[0] += 1
            vp, vs, rho, _ = mat_update(self.vp, self.vs, self.rho, *d, eps, self.limits, it, self.inv_iter,
                                        self.scalerho)
            return self.misfit((vp, vs, rho))

        eps, L2t, epst, found = step_length(objective, L2, self.eps_scale, self.scalefac, self.stepmax)
        # FWI_PSV.c:686-694: no update after a failed search once MIN_ITER iterations are done;
        # before that the smallest step tried is taken
        if it > min_iter and not found:
            eps = 0.0
        self.vp, self.vs, self.rho, _ = mat_update(self.vp, self.vs, self.rho, *d, eps, self.limits, it,
                                                   self.inv_iter, self.scalerho)
        if self.inv_modelfile is not None and self.rank0:
            write_inv_model(self.inv_modelfile, (self.vp, self.vs, self.rho))
        t3 = time.perf_counter()
        self.history.append({"iteration": it, "misfit": L2, "eps": eps, "L2t": L2t, "epst": epst, "found": found,
                             "gradient_s": t1 - t0, "optimizer_s": t2 - t1, "step_search_s": t3 - t2,
                             "test_models": ntests[0]})
        return L2

    def close(self):
        if self.own_optimizer and self.optimizer is not None:
            self.optimizer.close()
        self.optimizer = None
        if self.precond is not None:
            self.precond.close()
            self.precond = None


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
