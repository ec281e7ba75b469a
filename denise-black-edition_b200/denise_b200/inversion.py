"""The reference's main program for a parameter file and, for FWI, a workflow
file (src/denise.c: ``denise <par.inp> <workflow.inp>``).

MODE 0 is the forward modelling of FD_PSV (the native driver, dn_forward_inp).
MODE 1 is the FWI of FWI_PSV.c for the P-SV path:

* starting model MFILE.{vp,vs,rho} (READMOD 1); sources from SOURCE_FILE, one
  shot per line, firing that source or, with RUN_MULTIPLE_SHOTS 0, all of them
  (count_src.c); receivers REC_FILE.dat (READREC 1);
* per shot the wavelets of wavelet.c for the stage's N_ORDER, the QUELLART 6
  spike band-limited by ORDER_SPIKE / FC_SPIKE_2 / FC_SPIKE_1 and, in stages
  with TIME_FILT, both sources and data band-limited by ORDER / FC / FC_START
  (grad_obj_psv.c:136-156);
* observed data DATA_DIR_x.su.shot<n> and DATA_DIR_y.su.shot<n> (inseis.c);
* the misfit and the step-length tests over the test shots TESTSHOT_START ..
  TESTSHOT_END by TESTSHOT_INCR (grad_obj_psv.c:179, obj_psv.c:50);
* gradient conditioning from SWS_TAPER_GRAD_VERT / _HOR / _SOURCES, GRADT1-4,
  EXP_TAPER_GRAD_HOR, the per-shot circular taper (SWS_TAPER_CIRCULAR_PER_SHOT,
  SRTSHAPE, SRTRADIUS, FILTSIZE) and the stage's SPATFILTER;
* model bounds VP/VS/RHO UPPER/LOWERLIM, the reference's optimisers (GRAD_METHOD
  2: L-BFGS with NLBFGS pairs; 1: PCG with PCG_BETA) on gradients normalised by
  the starting model's averages, step search EPS_SCALE / STEPMAX / SCALEFAC,
  ITERMAX and MIN_ITER per stage;
* outputs as FWI_PSV.c writes them: the model after every update,
  INV_MODELFILE_{vp,vs,rho}.bin (calc_mat_change_test_PSV.c); after every
  L-BFGS step the JACOBIAN files <JACOBIAN>_{p,p_u,p_rho,p_vp,p_vs,p_mrho,c,
  c_u,c_rho}.old (extract_LBFGS_PSV.c); with INV_MOD_OUT 0 the model of a stage
  that ends by the abort criterion or a failed step search,
  INV_MODELFILE_{vp,vs,rho}_stage_<n>.bin (model_freq_out_PSV.c); with
  INV_MOD_OUT 1 the model after every iteration,
  INV_MODELFILE_{vp,vs,rho}_stage_<n>_it_<iter>.bin (model_it_out_PSV.c); and
  the MISFIT_LOG_FILE lines.

Switches the GPU path does not provide raise NotImplementedError (
SWS_TAPER_FILE, TRKILL, TIMELAPSE, gravity, and the workflow options listed in
workflow.py).  Run as ``python -m denise_b200 <par.inp> [<workflow.inp>] [device]``.
"""
import os

import numpy as np

from . import _lib, io
from .api import PsvParams, tdfilt, wavelet


def params_from_inp(inp, ts, **kw):
    """PsvParams of a parameter file (dn_inp_params), with overrides."""
    c = io.inp_params(inp, ts)
    d = {}
    for name in PsvParams.__dataclass_fields__:
        if name == "fl":
            d[name] = tuple(float(c.fl[k]) for k in range(c.L))
        elif hasattr(c, name):
            d[name] = getattr(c, name)
    d.update(kw)
    return PsvParams(**d)


def _check_supported(inp):
    if inp.physics != 1:
        raise NotImplementedError(f"PHYSICS={inp.physics}: only 2-D P-SV (1) is built")
    if inp.readmod != 1 or inp.srcrec != 1 or inp.readrec not in (1, 2):
        raise NotImplementedError("READMOD and SRCREC must be 1 (model and source files), READREC 1 or 2 "
                                  "(one receiver file or one per shot)")
    for key, what in (("sws_taper_file", "SWS_TAPER_FILE"), ("trkill", "TRKILL"), ("timelapse", "TIMELAPSE"),
                      ("gravity", "GRAVITY")):
        if inp.get(key):
            raise NotImplementedError(f"{what} is not provided")


class Acquisition:
    """Sources, receivers and per-shot wavelets of a parameter file."""

    def __init__(self, inp, device=0):
        self.inp = inp
        self.device = device
        self.srcpos, self.ts = io.read_sources(inp.get("source_file"))
        self.rec_i, self.rec_j = io.read_receivers(inp.get("rec_file") + ".dat", list(inp.refrec), inp.dh) \
            if inp.readrec != 2 else (None, None)
        self.shot_receivers = {}
        self.nt = io.inp_nt(inp)
        self.nshots = len(self.srcpos)
        self.file_signals = {}

    def shot(self, k, n_order=0):
        """Shot k (0-based) as an FWI shot tuple, wavelets integrated n_order times."""
        inp, nt = self.inp, self.nt
        idx = [k] if inp.run_multiple_shots else list(range(self.nshots))
        sig = None
        if inp.quellart == 3:
            if k not in self.file_signals:
                self.file_signals[k] = io.read_signal_file(f"{inp.get('signal_file')}_shot_{k + 1}.dat")
            sig = self.file_signals[k]
        si, sj, types, azi, sigs = [], [], [], [], []
        for l in idx:
            s = self.srcpos[l]
            i, j = io.source_cell(float(s[0]), float(s[1]), inp.dh)
            if not (1 <= i <= inp.nx and 1 <= j <= inp.ny):   # splitsrc.c on one rank: not injected
                continue
            si.append(i)
            sj.append(j)
            types.append(int(s[7]))
            azi.append(float(s[6]))
            sigs.append(wavelet(inp.quellart, nt, inp.dt, float(s[3]), float(s[4]), float(s[5]), n_order,
                                fc_spike_1=inp.fc_spike_1, fc_spike_2=inp.fc_spike_2, ts=self.ts, signal=sig))
        if not si:
            raise ValueError(f"shot {k + 1}: no source inside the grid")
        signals = np.stack(sigs).astype(np.float32)
        if inp.quellart == 6:
            signals = tdfilt(signals, inp.dt, inp.order_spike, inp.fc_spike_2, inp.fc_spike_1, self.device)
        s0 = self.srcpos[k]
        ri, rj = self.receivers(k)
        return (np.array(si, np.int32), np.array(sj, np.int32), signals, ri, rj,
                np.array(types, np.int32), np.array(azi, np.float32), (float(s0[0]), float(s0[1])))

    def receivers(self, k):
        """Receivers of shot k (0-based): REC_FILE.dat, or REC_FILE_shot_<k+1>.dat with
        READREC 2 (receiver.c:32-41, read per shot by grad_obj_psv.c and obj_psv.c)."""
        if self.inp.readrec != 2:
            return self.rec_i, self.rec_j
        if k not in self.shot_receivers:
            self.shot_receivers[k] = io.read_receivers(f"{self.inp.get('rec_file')}_shot_{k + 1}.dat",
                                                       list(self.inp.refrec), self.inp.dh)
        return self.shot_receivers[k]

    def test_shots(self):
        """0-based indices of TESTSHOT_START .. TESTSHOT_END by TESTSHOT_INCR."""
        a, b, c = self.inp.testshot[1], self.inp.testshot[2], max(self.inp.testshot[3], 1)
        return [k - 1 for k in range(1, self.nshots + 1) if a <= k <= b and (k - a) % c == 0]


def read_observed(inp, nshots, ntr, nt):
    """DATA_DIR_x.su.shot<n> and DATA_DIR_y.su.shot<n> (inseis.c) of every shot; ntr is
    the receiver count, or a function of the 0-based shot giving it (READREC 2)."""
    base = inp.get("data_dir")
    count = ntr if callable(ntr) else (lambda k: ntr)
    return [(io.read_su(f"{base}_x.su.shot{k}", count(k - 1), nt), io.read_su(f"{base}_y.su.shot{k}", count(k - 1), nt))
            for k in range(1, nshots + 1)]


def precond_base(inp, acq):
    """PrecondConfig of the parameter file's taper switches (None when all are off)."""
    from .precond import PrecondConfig

    if not (inp.sws_taper_grad_vert or inp.sws_taper_grad_hor or inp.sws_taper_grad_sources):
        return None
    return PrecondConfig(taper_vert=inp.sws_taper_grad_vert, taper_hor=inp.sws_taper_grad_hor,
                         taper_sources=inp.sws_taper_grad_sources, gradt=tuple(int(x) for x in inp.gradt[1:5]),
                         exp_taper_grad_hor=inp.exp_taper_grad_hor, srtshape=inp.srtshape, srtradius=inp.srtradius,
                         filtsize=inp.filtsize,
                         sources=[(float(s[0]), float(s[1])) for s in acq.srcpos],
                         receivers=list(zip(*[np.concatenate([acq.receivers(k)[c] for k in range(acq.nshots)]).tolist()
                                              for c in (0, 1)])) if inp.readrec == 2
                         else list(zip(acq.rec_i.tolist(), acq.rec_j.tolist())))


def fwi_inp(par_path, workflow_path, device=0, snap_precision=_lib.SNAP_F32, dist=None, resume=False):
    """MODE 1 of a parameter file with its workflow file; returns run_workflow's
    (vp, vs, rho, [StageResult]).  Paths inside the files are relative to the
    current directory, as in the reference."""
    from .workflow import read_workflow, run_workflow

    inp = io.read_inp(par_path)
    if inp.mode != 1:
        raise ValueError(f"{par_path}: MODE={inp.mode}; fwi_inp runs MODE 1")
    _check_supported(inp)
    acq = Acquisition(inp, device)
    p = params_from_inp(inp, acq.ts, store_snapshots=1, snap_precision=snap_precision)
    nx, ny = p.nx, p.ny
    model = [io.read_model_file(f"{inp.get('mfile')}.{ext}", nx, ny) for ext in ("vp", "vs", "rho")]
    if p.L:
        model += [io.read_model_file(f"{inp.get('mfile')}.{ext}", nx, ny) for ext in ("qp", "qs")]
    obs = read_observed(inp, acq.nshots, lambda k: len(acq.receivers(k)[0]), p.nt)
    stages = read_workflow(workflow_path)
    limits = (inp.vplowerlim, inp.vpupperlim, inp.vslowerlim, inp.vsupperlim, inp.rholowerlim, inp.rhoupperlim)
    shot_taper = (inp.srtshape, inp.srtradius, inp.filtsize) if inp.sws_taper_circular_per_shot else None
    out_prefix = inp.get("inv_modelfile") or None
    misfit_log = inp.get("misfit_log_file") or None
    for path in (out_prefix, misfit_log, inp.get("jacobian") or None):
        d = os.path.dirname(path) if path else ""
        if d:
            os.makedirs(d, exist_ok=True)
    return run_workflow(p, model, None, obs, limits, stages, itermax=inp.itermax, min_iter=inp.min_iter,
                        precond_base=precond_base(inp, acq), shot_taper=shot_taper, device=device, dist=dist,
                        out_prefix=out_prefix, misfit_log=misfit_log, resume=resume, inv_mod_out=inp.inv_mod_out,
                        shots_for_stage=lambda st: [acq.shot(k, st["N_ORDER"]) for k in range(acq.nshots)],
                        grad_method=inp.grad_method, nlbfgs=inp.nlbfgs or 20, pcg_beta=inp.pcg_beta or 2,
                        jacobian=inp.get("jacobian") or None, eps_scale=inp.eps_scale, scalefac=inp.scalefac,
                        stepmax=inp.stepmax, test_shots=acq.test_shots())


def main(argv=None):
    import sys

    argv = sys.argv[1:] if argv is None else argv
    if not argv or argv[0] in ("-h", "--help"):
        print("usage: python -m denise_b200 <par.inp> [<workflow.inp>] [device]")
        return 2
    inp = io.read_inp(argv[0])
    rest = list(argv[1:])
    device = int(rest.pop()) if rest and rest[-1].isdigit() else 0
    if inp.mode == 0:
        io.forward_inp(argv[0], device)
        return 0
    if inp.mode == 1:
        if not rest:
            print("MODE 1 needs the workflow file: python -m denise_b200 <par.inp> <workflow.inp>")
            return 2
        _, _, _, results = fwi_inp(argv[0], rest[0], device)
        for r in results:
            print(f"stage {r.stage}: {r.iterations} iterations ({r.reason}), misfits {r.misfits}")
        return 0
    print(f"MODE={inp.mode}: forward modelling (0) and FWI (1) are provided")
    return 2
