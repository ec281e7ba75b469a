"""Multi-stage FWI workflow: the stage loop of FWI_PSV.c:398-840 driven by a
workflow file in the reference's format (read_par_inv.c).

A workflow file holds one header line of 30 names and one line of 30 values
per stage, read with fscanf, so line breaks inside a stage do not matter; the
number of stages is the number of newlines minus one (FWI_PSV.c:157-163).
Each stage configures the inversion: time-domain filter (TIME_FILT, ORDER,
FC_START, FC_END), objective (LNORM, N_ORDER, OFFSET_MUTE, OFFSETC, TIMEWIN 5
with GAMMA and TWLENGTH_MINUS), smoothing (SPATFILTER, WD_DAMP, WD_DAMP1),
energy preconditioning (EPRECOND 1 or 3, with C_vp, C_vs, C_rho the averages
of the starting model, FWI_PSV.c:538-580) and the iterations from which vp, vs
and rho are inverted (INV_*_ITER), and it runs until the misfit of the last
iteration differs from the one two iterations earlier by at most PRO
(relative) after MIN_ITER iterations, or the step search fails, or ITERMAX
iterations ran (FWI_PSV.c:784-830).  The L-BFGS history is cleared between
stages.  Options the GPU path does not provide raise NotImplementedError:
ROWI, INV_STF, NORMALIZE, ENV (LNORM 6), GAMMA_GRAV and TIMEWIN 1-4; Qs
(INV_QS_ITER) is not inverted.  Each stage's model can be written as
model_freq_out_PSV.c names it and the misfit log as FWI_PSV.c writes it, and
a run can resume after the last stage whose model files exist.
"""
import dataclasses

import numpy as np

STAGE_KEYS = ("PRO", "TIME_FILT", "FC_START", "FC_END", "ORDER", "TIMEWIN", "GAMMA", "TWLENGTH_MINUS",
              "TWLENGTH_PLUS", "INV_VP_ITER", "INV_VS_ITER", "INV_RHO_ITER", "INV_QS_ITER", "SPATFILTER", "WD_DAMP",
              "WD_DAMP1", "EPRECOND", "LNORM", "ROWI", "INV_STF", "OFFSETC_STF", "EPS_STF", "NORMALIZE",
              "OFFSET_MUTE", "OFFSETC", "SCALERHO", "SCALEQS", "ENV", "GAMMA_GRAV", "N_ORDER")
INT_KEYS = {"TIME_FILT", "ORDER", "TIMEWIN", "INV_VP_ITER", "INV_VS_ITER", "INV_RHO_ITER", "INV_QS_ITER",
            "SPATFILTER", "EPRECOND", "LNORM", "ROWI", "INV_STF", "NORMALIZE", "OFFSET_MUTE", "ENV", "N_ORDER"}


def _c_int(tok):
    """fscanf %i: decimal, 0x hexadecimal or 0 octal, with an optional sign."""
    t = tok.strip()
    sign = -1 if t.startswith("-") else 1
    t = t.lstrip("+-")
    if t.lower().startswith("0x"):
        return sign * int(t, 16)
    if len(t) > 1 and t.startswith("0"):
        return sign * int(t, 8)
    return sign * int(t)


def read_workflow(path):
    """The stages of a workflow file as a list of dicts keyed by STAGE_KEYS.  As
    read_par_inv's fscanf does, a stage whose values run out (more newlines than
    stage lines, e.g. a stage broken over two lines) keeps the values of the stage
    before it for the keys it could not read."""
    text = open(path).read()
    nstages = text.count("\n") - 1
    tok = text.split()
    n = len(STAGE_KEYS)
    if nstages < 1 or len(tok) < 2 * n:
        raise ValueError(f"{path}: {len(tok)} values, {nstages} stages of {n}")
    stages, cur, pos = [], {key: 0 for key in STAGE_KEYS}, n
    for _ in range(nstages):
        cur = dict(cur)
        for key in STAGE_KEYS:
            if pos >= len(tok):
                break
            cur[key] = _c_int(tok[pos]) if key in INT_KEYS else float(tok[pos])
            pos += 1
        stages.append(cur)
    return stages


def model_averages(vp, vs, rho):
    """C_vp, C_vs, C_rho of FWI_PSV.c:538-580: float sums in the reference's loop order
    (x outer, depth inner = file order) divided by NX*NY."""
    out = []
    for a in (vp, vs, rho):
        a = np.ascontiguousarray(a, np.float32)
        total = np.cumsum(a.ravel(), dtype=np.float32)[-1]
        out.append(float(np.float32(total / np.float32(a.size))))
    return tuple(out)


@dataclasses.dataclass
class StageResult:
    stage: int
    iterations: int
    misfits: list
    reason: str


def _check_supported(st, params):
    for key in ("ROWI", "INV_STF", "NORMALIZE", "ENV"):
        if st[key]:
            raise NotImplementedError(f"{key} = {st[key]} is not provided by the GPU path")
    if st["GAMMA_GRAV"]:
        raise NotImplementedError("joint gravity inversion (GAMMA_GRAV) is not provided")
    if st["TIMEWIN"] not in (0, 5):
        raise NotImplementedError(f"TIMEWIN {st['TIMEWIN']} (picked-time windows) is not provided")
    if st["LNORM"] == 6:
        raise NotImplementedError("LNORM 6 (envelope misfit) needs a Hilbert transform")
    if st["EPRECOND"] not in (0, 1, 3):
        raise NotImplementedError(f"EPRECOND {st['EPRECOND']} is not provided")


def stage_fwi(params, model, shots, obs, limits, st, averages, precond_base=None, shot_taper=None, device=0,
              nlbfgs=20, eps_scale=0.01, scalefac=2.0, stepmax=4, dist=None, test_shots=None, grad_method=2,
              pcg_beta=2, optimizer=None, jacobian=None, inv_modelfile=None):
    """An fwi.FWI configured by one workflow stage."""
    from . import fwi
    from .precond import PrecondConfig

    _check_supported(st, params)
    p = params.replace(eprecond=st["EPRECOND"])
    time_filter = None
    if st["TIME_FILT"]:
        time_filter = (st["ORDER"], st["FC_END"], st["FC_START"] if st["FC_START"] > 0 else 0.0)
    residual = {"lnorm": st["LNORM"], "grad_form": p.grad_form, "n_order": st["N_ORDER"],
                "offset_mute": st["OFFSET_MUTE"], "offsetc": st["OFFSETC"], "timewin": st["TIMEWIN"],
                "gamma": st["GAMMA"], "twlength_minus": st["TWLENGTH_MINUS"]}
    precond = None
    if st["SPATFILTER"] or precond_base is not None:
        base = precond_base if precond_base is not None else PrecondConfig()
        precond = dataclasses.replace(base, spatfilter=st["SPATFILTER"], wd_damp=st["WD_DAMP"],
                                      wd_damp1=st["WD_DAMP1"], fc_end=st["FC_END"],
                                      c_vs=averages[1] if not base.c_vs else base.c_vs)
    energy = averages if st["EPRECOND"] in (1, 3) else None
    return fwi.FWI(p, model, shots, obs, limits, device=device, nlbfgs=nlbfgs, eps_scale=eps_scale,
                   scalefac=scalefac, stepmax=stepmax, dist=dist, precond=precond, shot_taper=shot_taper,
                   time_filter=time_filter, residual=residual, energy=energy,
                   inv_iter=(st["INV_VP_ITER"], st["INV_VS_ITER"], st["INV_RHO_ITER"]), test_shots=test_shots,
                   grad_method=grad_method, pcg_beta=pcg_beta, averages=averages, optimizer=optimizer,
                   jacobian=jacobian, inv_modelfile=inv_modelfile, scalerho=st["SCALERHO"])


def stage_files(prefix, stage):
    """The model files model_freq_out_PSV.c writes at the end of a stage:
    <INV_MODELFILE>_{vp,vs,rho}_stage_<n>.bin, x-major float32."""
    return tuple(f"{prefix}_{name}_stage_{stage}.bin" for name in ("vp", "vs", "rho"))


def _write_log(path, f, st, stage):
    """The misfit log line of FWI_PSV.c:734-743 (MISFIT_LOG_FILE): opteps, epst1[1..3],
    L2t[1..4] and the stage, with FC_START and FC before the stage when TIME_FILT is set."""
    h = f.history[-1]
    eps = h["eps"]          # opteps_vp: the step taken (0 after a failed search past MIN_ITER)
    L2t = list(h["L2t"]) + [h["misfit"]]
    epst = list(h["epst"])
    v = (eps, epst[0], epst[1], epst[2], L2t[0], L2t[1], L2t[2], L2t[3])
    with open(path, "a") as fp:
        if st["TIME_FILT"] == 0:
            fp.write("%e \t %e \t %e \t %e \t %e \t %e \t %e \t %e \t %d \n" % (v + (stage,)))
        else:
            fp.write("%e \t %e \t %e \t %e \t %e \t %e \t %e \t %e \t %f \t %f \t %d \n"
                     % (v + (st["FC_START"], st["FC_END"], stage)))


def iteration_files(prefix, stage, it):
    """The model files model_it_out_PSV.c writes after every iteration (INV_MOD_OUT 1):
    <INV_MODELFILE>_{vp,vs,rho}_stage_<n>_it_<iter>.bin."""
    return tuple(f"{prefix}_{name}_stage_{stage}_it_{it}.bin" for name in ("vp", "vs", "rho"))


def _write_model(files, model):
    for a, x in zip(model, files):
        np.ascontiguousarray(a, np.float32).tofile(x)


def run_workflow(params, model, shots, obs, limits, stages, itermax, min_iter=0, precond_base=None,
                 shot_taper=None, device=0, dist=None, out_prefix=None, misfit_log=None, resume=False,
                 shots_for_stage=None, inv_mod_out=None, grad_method=2, nlbfgs=20, pcg_beta=2, jacobian=None,
                 **fwi_kw):
    """Runs the stages in order from the starting model; returns (vp, vs, rho, [StageResult]).

    The loop is FWI_PSV.c:398-840: the model averages C_vp, C_vs, C_rho of the
    starting model normalise the gradients of every stage; one optimiser
    (grad_method 2: L-BFGS with nlbfgs pairs, 1: PCG with pcg_beta) serves all
    stages and is reset only when a stage ends by its abort criterion; a stage
    ends after ITERMAX iterations or, once MIN_ITER iterations are done, when
    the misfit changed by at most PRO over two iterations or the step search
    failed (a failed search moves the model by 0 after MIN_ITER iterations and
    by the smallest step tried before).

    shots_for_stage: a function of the stage's dict returning its shots, for
    wavelets that depend on the stage (wavelet.c integrates N_ORDER times);
    otherwise every stage uses `shots`.

    out_prefix: the INV_MODELFILE prefix: each update writes <prefix>_{vp,vs,rho}.bin
    (calc_mat_change_test_PSV) and the stage models as below (rank 0 of dist).
    inv_mod_out: None writes every stage's final model; 0 or 1 follow FWI_PSV.c: 0 writes
    a stage's model only when the stage ends by the abort criterion or a failed step
    search (model_freq_out_PSV), 1 writes the model after every iteration
    (iteration_files, model_it_out_PSV) and no stage files.
    jacobian: the JACOBIAN prefix of the L-BFGS files (extract_LBFGS_PSV).
    misfit_log: append one line per iteration in the reference's misfit-log format.
    resume: start after the last stage whose three model files exist, from that model (the
    reference's restart from its last written model)."""
    from .fwi import Optimizer

    vp, vs, rho = [np.ascontiguousarray(a, np.float32) for a in model[:3]]
    averages = model_averages(vp, vs, rho)          # of the starting model (iter_true == 1)
    nx, ny = params.nx, params.ny
    rank0 = dist is None or not dist.is_initialized() or dist.get_rank() == 0
    results, first = [], 1
    if misfit_log is not None and rank0 and not resume:
        open(misfit_log, "w").close()   # FWI_PSV.c:586-589: opened with "w" at the first iteration
    if resume and out_prefix is not None:
        import os

        for k in range(len(stages), 0, -1):
            files = stage_files(out_prefix, k)
            if all(os.path.exists(x) for x in files):
                vp, vs, rho = [np.fromfile(x, np.float32, nx * ny).reshape(nx, ny) for x in files]
                results = [StageResult(j, 0, [], "resumed") for j in range(1, k + 1)]
                first = k + 1
                break
    optimizer = Optimizer(grad_method, nx, ny, nlbfgs, pcg_beta, device)
    try:
        for k in range(first, len(stages) + 1):
            st = stages[k - 1]
            sh = shots_for_stage(st) if shots_for_stage is not None else shots
            f = stage_fwi(params, (vp, vs, rho), sh, obs, limits, st, averages, precond_base, shot_taper, device,
                          dist=dist, nlbfgs=nlbfgs, grad_method=grad_method, pcg_beta=pcg_beta,
                          optimizer=optimizer, jacobian=jacobian, inv_modelfile=out_prefix, **fwi_kw)
            misfits, reason, it = [], "ITERMAX", 0
            try:
                for it in range(1, itermax + 1):
                    misfits.append(f.iterate(it, min_iter))
                    if misfit_log is not None and rank0:
                        _write_log(misfit_log, f, st, k)
                    found = f.history[-1]["found"]
                    stop = None
                    # FWI_PSV.c:782-832 (the reference reads L2_hist[iter - 2] before it exists in
                    # iterations 1 and 2, where the criterion cannot hold)
                    if it > min_iter:
                        if it >= 3 and abs(misfits[-3] - misfits[-1]) / misfits[-3] <= st["PRO"]:
                            stop = "PRO"
                        elif not found:
                            stop = "step search failed"
                    if stop is not None:
                        reason = stop
                        if out_prefix is not None and rank0 and inv_mod_out == 0:
                            _write_model(stage_files(out_prefix, k), (f.vp, f.vs, f.rho))
                        optimizer.reset()
                        break
                    if out_prefix is not None and rank0 and inv_mod_out == 1:
                        _write_model(iteration_files(out_prefix, k, it), (f.vp, f.vs, f.rho))
            finally:
                f.close()
            vp, vs, rho = f.vp, f.vs, f.rho
            if out_prefix is not None and rank0 and inv_mod_out is None:
                _write_model(stage_files(out_prefix, k), (vp, vs, rho))
            results.append(StageResult(k, it, misfits, reason))
    finally:
        optimizer.close()
    return vp, vs, rho, results
