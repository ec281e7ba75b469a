"""Writes DENISE parameter files (.inp) and the data files they name, for the
host I/O tests and the command-line parity tests.

The .inp layout is positional: after a first line that is never read, every
line that does not start with '#' is the next parameter, in the order of the
reference's read_par (src/read_par.c).  The key text before '=' is free (it is
scanned and discarded); the keys written here are this project's own.
"""
import os

import numpy as np

# (line number order) name, kind: i int, f float, s string, fl float list, f2 "a , b", i3 / i4 "a, b, c[, d]"
LINES = [
    ("MODE", "i"), ("PHYSICS", "i"), ("NPROCX", "i"), ("NPROCY", "i"), ("FDORDER", "i"), ("MAXRELERROR", "i"),
    ("NX", "i"), ("NY", "i"), ("DH", "f"), ("TIME", "f"), ("DT", "f"), ("QUELLART", "i"), ("SIGNAL_FILE", "s"),
    ("TS", "f"), ("SRCREC", "i"), ("SOURCE_FILE", "s"), ("RUN_MULTIPLE_SHOTS", "i"), ("FC_SPIKE_1", "f"),
    ("FC_SPIKE_2", "f"), ("ORDER_SPIKE", "i"), ("WRITE_STF", "i"), ("READMOD", "i"), ("MFILE", "s"),
    ("WRITEMOD", "i"), ("L", "i"), ("FL", "fl"), ("TAU", "f"), ("FREE_SURF", "i"), ("FW", "i"), ("DAMPING", "f"),
    ("FPML", "f"), ("NPOWER", "f"), ("K_MAX_PML", "f"), ("BOUNDARY", "i"), ("SNAP", "i"), ("SNAP_SHOT", "i"),
    ("TSNAP1", "f"), ("TSNAP2", "f"), ("TSNAPINC", "f"), ("IDX", "i"), ("IDY", "i"), ("SNAP_FORMAT", "i"),
    ("SNAP_FILE", "s"), ("SEISMO", "i"), ("READREC", "i"), ("REC_FILE", "s"), ("REFREC", "f2"),
    ("N_STREAMER", "i"), ("REC_INCR_X", "f"), ("REC_INCR_Y", "f"), ("NDT", "i"), ("SEIS_FORMAT", "i"),
    ("SEIS_FILE_VX", "s"), ("SEIS_FILE_VY", "s"), ("SEIS_FILE_CURL", "s"), ("SEIS_FILE_DIV", "s"),
    ("SEIS_FILE_P", "s"), ("LOG_FILE", "s"), ("LOG", "i"), ("ITERMAX", "i"), ("JACOBIAN", "s"), ("DATA_DIR", "s"),
    ("TAPER", "i"), ("TAPERLENGTH", "i"), ("GRADT", "i4"), ("INVMAT1", "i"), ("GRAD_FORM", "i"),
    ("QUELLTYPB", "i"), ("TESTSHOT", "i3"), ("SWS_TAPER_GRAD_VERT", "i"), ("SWS_TAPER_GRAD_HOR", "i"),
    ("EXP_TAPER_GRAD_HOR", "f"), ("SWS_TAPER_GRAD_SOURCES", "i"), ("SWS_TAPER_CIRCULAR_PER_SHOT", "i"),
    ("SRTSHAPE", "i"), ("SRTRADIUS", "f"), ("FILTSIZE", "i"), ("SWS_TAPER_FILE", "i"), ("TFILE", "s"),
    ("INV_MOD_OUT", "i"), ("INV_MODELFILE", "s"), ("VPUPPERLIM", "f"), ("VPLOWERLIM", "f"), ("VSUPPERLIM", "f"),
    ("VSLOWERLIM", "f"), ("RHOUPPERLIM", "f"), ("RHOLOWERLIM", "f"), ("QSUPPERLIM", "f"), ("QSLOWERLIM", "f"),
    ("GRAD_METHOD", "i"), ("PCG_BETA", "i"), ("NLBFGS", "i"), ("MODEL_FILTER", "i"), ("FILT_SIZE", "i"),
    ("DTINV", "i"), ("EPS_SCALE", "f"), ("STEPMAX", "i"), ("SCALEFAC", "f"), ("TRKILL", "i"),
    ("TRKILL_FILE", "s"), ("PICKS_FILE", "s"), ("MISFIT_LOG_FILE", "s"), ("MIN_ITER", "i"), ("GRAD_FILTER", "i"),
    ("FILT_SIZE_GRAD", "i"), ("TIMELAPSE", "i"), ("DATA_DIR_T0", "s"), ("RTMOD", "i"), ("GRAVITY", "i"),
    ("NGRAVB", "i"), ("NZGRAV", "i"), ("GRAV_TYPE", "i"), ("BACK_DENSITY", "i"), ("DFILE", "s"), ("RTM_SHOT", "i"),
]

DEFAULTS = dict(
    MODE=0, PHYSICS=1, NPROCX=1, NPROCY=1, FDORDER=8, MAXRELERROR=1, NX=120, NY=80, DH=5.0, TIME=0.12, DT=4e-4,
    QUELLART=1, SIGNAL_FILE="wavelet/none", TS=8.0, SRCREC=1, SOURCE_FILE="source/sources.dat", RUN_MULTIPLE_SHOTS=1,
    FC_SPIKE_1=-5.0, FC_SPIKE_2=15.0, ORDER_SPIKE=5, WRITE_STF=0, READMOD=1, MFILE="model/test", WRITEMOD=0, L=0,
    FL=[5.0], TAU=0.0, FREE_SURF=1, FW=10, DAMPING=1500.0, FPML=10.0, NPOWER=4.0, K_MAX_PML=1.0, BOUNDARY=0, SNAP=0,
    SNAP_SHOT=1, TSNAP1=0.002, TSNAP2=0.1, TSNAPINC=0.1, IDX=1, IDY=1, SNAP_FORMAT=3, SNAP_FILE="snap/test",
    SEISMO=1, READREC=1, REC_FILE="receiver/receivers", REFREC=[0.0, 0.0], N_STREAMER=0, REC_INCR_X=0.0,
    REC_INCR_Y=0.0, NDT=1, SEIS_FORMAT=1, SEIS_FILE_VX="su/test_x.su", SEIS_FILE_VY="su/test_y.su",
    SEIS_FILE_CURL="su/test_rot.su", SEIS_FILE_DIV="su/test_div.su", SEIS_FILE_P="su/test_p.su",
    LOG_FILE="log/test.log", LOG=0, ITERMAX=1, JACOBIAN="jacobian/gradient", DATA_DIR="su/obs", TAPER=0,
    TAPERLENGTH=4, GRADT=[1, 2, 3, 4], INVMAT1=1, GRAD_FORM=1, QUELLTYPB=1, TESTSHOT=[1, 1, 1], GRAD_METHOD=2,
    NLBFGS=20, DTINV=2, EPS_SCALE=0.01, STEPMAX=4, SCALEFAC=2.0,
)


def _fmt(kind, v):
    if kind == "i":
        return str(int(v)) if not isinstance(v, str) else v
    if kind == "f":
        return repr(float(v)) if not isinstance(v, str) else v
    if kind == "s":
        return str(v)
    if kind == "fl":
        return " ".join(repr(float(x)) for x in v)
    if kind == "f2":
        return f"{float(v[0])!r} , {float(v[1])!r}"
    return ", ".join(str(int(x)) for x in v)


def write_inp(path, blank_after=None, stray_after=None, comments=True, **values):
    """A parameter file with every line of the reference's layout; `values`
    override DEFAULTS (a string value is written verbatim, e.g. a hex int).
    blank_after=k adds an empty line after parameter k (the reader's scan skips
    it); stray_after=k adds a line that is not a comment (it becomes a parameter
    line and shifts every later value by one)."""
    vals = dict(DEFAULTS)
    vals.update(values)
    out = ["#-------- parameter file (header line, never read)"]
    for k, (name, kind) in enumerate(LINES, start=1):
        if comments and k % 7 == 1:
            out.append(f"# ---- block {k} ----")
        v = vals.get(name, 0 if kind in ("i",) else 0.0 if kind == "f" else "none" if kind == "s" else
                     [0.0] if kind == "fl" else [0.0, 0.0] if kind == "f2" else [0, 0, 0, 0] if kind == "i4"
                     else [0, 0, 0])
        out.append(f"{name}_({name}) = {_fmt(kind, v)}")
        if blank_after == k:
            out.append("")
        if stray_after == k:
            out.append("stray_line = 7")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def write_case(root, nx=120, ny=80, dh=5.0, nshots=3, nrec=25, L=0, seed=0, src_cols=8, **inp):
    """A small forward-modelling case under `root`: models, sources, receivers
    and case.inp.  Returns the .inp path."""
    from denise_b200 import synth

    for d in ("model", "source", "receiver", "su", "log", "jacobian", "snap"):
        os.makedirs(os.path.join(root, d), exist_ok=True)
    vp, vs, rho = synth.base_model(nx, ny, dh, seed)
    files = {"vp": vp, "vs": vs, "rho": rho}
    if L:
        qp, qs = synth.q_model(nx, ny, seed)
        files.update(qp=qp, qs=qs)
    for ext, a in files.items():
        np.ascontiguousarray(a, np.float32).tofile(os.path.join(root, "model", f"test.{ext}"))
    xmax = (nx - 1) * dh
    with open(os.path.join(root, "source", "sources.dat"), "w") as f:
        f.write(f"{nshots}\n")
        for k in range(nshots):
            x = 0.25 * xmax + 0.5 * xmax * k / max(nshots - 1, 1)
            cols = [x, 0.0, 2 * dh, 0.0, 25.0, 1.0e3, 0.0, 1][:src_cols]
            f.write("\t".join(f"{c:.2f}" for c in cols) + "\n")
    with open(os.path.join(root, "receiver", "receivers.dat"), "w") as f:
        for k in range(nrec):
            f.write(f"{dh * 4 + (xmax - 8 * dh) * k / max(nrec - 1, 1):.3f}\t{3 * dh:.3f}\n")
    params = dict(NX=nx, NY=ny, DH=dh, L=L)
    if L:
        params["FL"] = [2.0, 8.0, 25.0][:L]
    params.update(inp)
    path = os.path.join(root, "case.inp")
    write_inp(path, **params)
    return path
