"""Host file I/O (include/denise_b200_io.h) against the reference's own readers
and writer, run from the reference build (oracle/_ref) in a separate process:
read_par, sources, receiver and outseis_glob.  CPU only."""
import ctypes
import os

import numpy as np
import pytest

import oracles as O
import inp_case
from denise_b200 import io

needs_ref = pytest.mark.skipif(not O.reference_available(), reason="reference build not present")

# -------------------------------------------------------------------------------------------------
# the reference's functions, each call in a fresh process (they set global state)
# -------------------------------------------------------------------------------------------------


def _ref_read_par(path):
    lib = ctypes.CDLL(O.REF_SO)
    iv = np.zeros(23, np.int32)
    fv = np.zeros(13, np.float32)
    strs = ctypes.create_string_buffer(74 * 8)
    assert lib.refh_read_par(path.encode(), O._ip(iv), O._fp(fv), strs) == 0
    names = [strs.raw[74 * k:74 * (k + 1)].split(b"\0")[0].decode() for k in range(8)]
    return iv, fv, names


def _ref_sources(root, path):
    # the reference keeps file names in 74-character buffers: run from the case directory
    os.chdir(root)
    lib = ctypes.CDLL(O.REF_SO)
    n = ctypes.c_int()
    sp = np.zeros(8 * 64, np.float32)
    ts = ctypes.c_float()
    lib.refh_sources(path.encode(), ctypes.byref(n), O._fp(sp), 64, ctypes.byref(ts))
    return sp[: 8 * n.value].reshape(n.value, 8), ts.value


def _ref_receivers(root, base, refx, refy, dh):
    os.chdir(root)
    lib = ctypes.CDLL(O.REF_SO)
    n = ctypes.c_int()
    ri = np.zeros(4096, np.int32)
    rj = np.zeros(4096, np.int32)
    lib.refh_receivers(base.encode(), ctypes.c_float(refx), ctypes.c_float(refy), ctypes.c_float(dh),
                       ctypes.byref(n), O._ip(ri), O._ip(rj), 4096)
    return ri[: n.value], rj[: n.value]


def _ref_outseis(path, sec, ri, rj, xs, ys, ndt, time, dt, dh, refx, refy):
    lib = ctypes.CDLL(O.REF_SO)
    sec = np.ascontiguousarray(sec, np.float32)
    ri = np.ascontiguousarray(ri, np.int32)
    rj = np.ascontiguousarray(rj, np.int32)
    f = ctypes.c_float
    assert lib.refh_outseis(path.encode(), O._fp(sec), sec.shape[0], sec.shape[1], O._ip(ri), O._ip(rj), f(xs), f(ys),
                            ndt, f(time), f(dt), f(dh), f(refx), f(refy)) == 0


# -------------------------------------------------------------------------------------------------
INT_FIELDS = ["mode", "physics", "nprocx", "nprocy", "fdorder", "maxrelerror", "nx", "ny", "quellart", "srcrec",
              "run_multiple_shots", "L", "free_surf", "fw", "boundary", "seismo", "readrec", "ndt", "seis_format",
              "invmat1", "grad_form", "quelltypb", "dtinv"]
FLT_FIELDS = ["dh", "time", "dt", "ts", "damping", "fpml", "npower", "k_max_pml"]
STR_FIELDS = ["source_file", "rec_file", "mfile", "seis_file_vx", "seis_file_vy", "seis_file_p", "signal_file",
              "jacobian"]

INP_VARIANTS = {
    "plain": dict(),
    "no-comments": dict(comments=False),
    "visco-fl-list": dict(L=3, FL=[2.0, 8.0, 25.0]),
    "hex-and-octal-ints": dict(NX="0x78", NY="0120", FDORDER="010"),
    "blank-line": dict(blank_after=20),
    "stray-line-shifts": dict(stray_after=20),
    "refrec-and-negative-fw": dict(REFREC=[12.5, -3.0], FW=-4),
}


@needs_ref
@pytest.mark.parametrize("name", list(INP_VARIANTS))
def test_inp_reader_matches_read_par(tmp_path, name):
    path = str(tmp_path / "p.inp")
    inp_case.write_inp(path, **INP_VARIANTS[name])
    ours = io.read_inp(path)
    iv, fv, strs = O.run_isolated(_ref_read_par, path)
    for k, f in enumerate(INT_FIELDS):
        assert ours.get(f) == int(iv[k]), f
    for k, f in enumerate(FLT_FIELDS):
        assert np.float32(ours.get(f)) == fv[k], f
    assert np.float32(ours.refrec[1]) == fv[8] and np.float32(ours.refrec[2]) == fv[9]
    for l in range(1, min(ours.L, 3) + 1):
        assert np.float32(ours.fl[l]) == fv[9 + l]
    for k, f in enumerate(STR_FIELDS):
        assert ours.get(f) == strs[k], f


def _ref_read_par_fwi(path):
    lib = ctypes.CDLL(O.REF_SO)
    iv = np.zeros(36, np.int32)
    fv = np.zeros(12, np.float32)
    strs = ctypes.create_string_buffer(74 * 8)
    assert lib.refh_read_par_fwi(path.encode(), O._ip(iv), O._fp(fv), strs) == 0
    names = [strs.raw[74 * k:74 * (k + 1)].split(b"\0")[0].decode() for k in range(8)]
    return iv, fv, names


FWI_INT = ["itermax", "taper", "taperlength", ("gradt", 1), ("gradt", 2), ("gradt", 3), ("gradt", 4),
           ("testshot", 1), ("testshot", 2), ("testshot", 3), "sws_taper_grad_vert", "sws_taper_grad_hor",
           "sws_taper_grad_sources", "sws_taper_circular_per_shot", "srtshape", "filtsize", "sws_taper_file",
           "inv_mod_out", "grad_method", "pcg_beta", "nlbfgs", "model_filter", "filt_size", "stepmax", "trkill",
           "min_iter", "grad_filter", "filt_size_grad", "timelapse", "rtmod", "gravity", "ngravb", "nzgrav",
           "grav_type", "back_density", "rtm_shot"]
FWI_FLT = ["exp_taper_grad_hor", "srtradius", "vpupperlim", "vplowerlim", "vsupperlim", "vslowerlim", "rhoupperlim",
           "rholowerlim", "qsupperlim", "qslowerlim", "eps_scale", "scalefac"]
FWI_STR = ["tfile", "inv_modelfile", "trkill_file", "picks_file", "misfit_log_file", "data_dir_t0", "dfile",
           "data_dir"]


@needs_ref
@pytest.mark.parametrize("name", ["plain", "stray-line-shifts"])
def test_inp_reader_inversion_lines_match_read_par(tmp_path, name):
    """Lines 60-115 (iterations, tapers, limits, L-BFGS, step search, logs) as read_par reads them."""
    path = str(tmp_path / "p.inp")
    kw = dict(INP_VARIANTS[name], MODE=1, ITERMAX=7, GRADT=[3, 9, 110, 140], TESTSHOT=[2, 5, 3], SWS_TAPER_GRAD_VERT=1,
              SWS_TAPER_GRAD_HOR=1, EXP_TAPER_GRAD_HOR=2.5, SWS_TAPER_GRAD_SOURCES=1, SWS_TAPER_CIRCULAR_PER_SHOT=1,
              SRTSHAPE=2, SRTRADIUS=12.5, FILTSIZE=3, INV_MODELFILE="model/inv", VPUPPERLIM=5500.0, VPLOWERLIM=1400.0,
              VSUPPERLIM=3300.0, VSLOWERLIM=0.0, RHOUPPERLIM=2800.0, RHOLOWERLIM=1000.0, NLBFGS=12, EPS_SCALE=0.02,
              STEPMAX=6, SCALEFAC=3.0, MISFIT_LOG_FILE="L2_LOG.dat", MIN_ITER=2, DATA_DIR="su/obs")
    inp_case.write_inp(path, **kw)
    ours = io.read_inp(path)
    iv, fv, strs = O.run_isolated(_ref_read_par_fwi, path)
    for k, f in enumerate(FWI_INT):
        got = getattr(ours, f[0])[f[1]] if isinstance(f, tuple) else ours.get(f)
        assert got == int(iv[k]), f
    for k, f in enumerate(FWI_FLT):
        assert np.float32(ours.get(f)) == fv[k], f
    for k, f in enumerate(FWI_STR):
        assert ours.get(f) == strs[k], f
    if name == "plain":
        assert ours.itermax == 7 and ours.nlbfgs == 12 and ours.get("misfit_log_file") == "L2_LOG.dat"


def test_inp_reader_known_values(tmp_path):
    """Without the reference: the positional semantics on a file this test writes."""
    path = str(tmp_path / "p.inp")
    inp_case.write_inp(path, NX="0x10", L=2, FL=[3.0, 9.0], FW=-1, REFREC=[1.5, 2.5], TIME=0.2, DT=4e-4)
    inp = io.read_inp(path)
    assert inp.nx == 16 and inp.L == 2 and list(inp.fl[1:3]) == [3.0, 9.0] and inp.fw == 0
    # the newline that ends the file, followed by EOF, also advances the counter (as in read_par)
    assert inp.lines == len(inp_case.LINES) + 1
    assert io.inp_nt(inp) == 500
    assert inp.get("source_file") == "source/sources.dat"
    assert list(inp.refrec[1:3]) == [1.5, 2.5]
    # an empty line is absorbed by the scan of the parameter line it starts
    inp_case.write_inp(path, blank_after=8)
    same = io.read_inp(path)
    assert same.lines == len(inp_case.LINES) + 1 and same.dh == 5.0
    # a line that is not a comment is a parameter line: every later value moves by one line
    inp_case.write_inp(path, stray_after=8)
    shifted = io.read_inp(path)
    assert shifted.lines == len(inp_case.LINES) + 2
    assert shifted.dh == 7.0 and shifted.time == 5.0


@needs_ref
@pytest.mark.parametrize("cols", [8, 7, 6])
def test_sources_match_reference(tmp_path, cols):
    root = str(tmp_path)
    inp_case.write_case(root, nshots=5, src_cols=cols)
    path = os.path.join(root, "source", "sources.dat")
    ours, ts = io.read_sources(path)
    ref, ref_ts = O.run_isolated(_ref_sources, root, "source/sources.dat")
    n = 8 if cols == 8 else 7   # with fewer than 8 columns the reference leaves the type unset
    np.testing.assert_array_equal(ours[:, :n], ref[:, :n])
    assert np.float32(ts) == np.float32(ref_ts)


@needs_ref
@pytest.mark.parametrize("ref_off", [(0.0, 0.0), (7.5, -2.5)])
def test_receivers_match_reference(tmp_path, ref_off):
    base = str(tmp_path / "rec")
    rng = np.random.default_rng(3)
    xs = np.concatenate([rng.uniform(-10, 500, 40), [100.0, 100.4, 250.0]])   # duplicates after rounding
    ys = np.concatenate([rng.uniform(0, 200, 40), [20.0, 20.1, 55.0]])
    with open(base + ".dat", "w") as f:
        for x, y in zip(xs, ys):
            f.write(f"{x:.3f} {y:.3f}\n")
    ri, rj = io.read_receivers(base + ".dat", [0.0, ref_off[0], ref_off[1], 0.0], 5.0)
    rri, rrj = O.run_isolated(_ref_receivers, str(tmp_path), "rec", ref_off[0], ref_off[1], 5.0)
    np.testing.assert_array_equal(ri, rri)
    np.testing.assert_array_equal(rj, rrj)
    assert len(ri) < len(xs)


@needs_ref
@pytest.mark.parametrize("ndt", [1, 3])
def test_su_writer_matches_outseis_glob(tmp_path, ndt):
    rng = np.random.default_rng(ndt)
    ntr, nt, dt, dh = 17, 300, 4e-4, 5.0
    time = np.float32(nt * dt)
    sec = rng.standard_normal((ntr, nt)).astype(np.float32)
    ri = np.arange(4, 4 + 3 * ntr, 3).astype(np.int32)
    rj = np.full(ntr, 5, np.int32)
    ours = str(tmp_path / "ours.su")
    ref = str(tmp_path / "ref.su")
    io.write_su(ours, sec, ndt, dt, time, dh, ri, rj, [0.0, 2.0, 1.0, 0.0], 312.5, 10.0)
    O.run_isolated(_ref_outseis, ref, sec, ri, rj, 312.5, 10.0, ndt, time, dt, dh, 2.0, 1.0)
    a = np.fromfile(ours, np.uint8)
    b = np.fromfile(ref, np.uint8)
    assert a.size == b.size
    ns = (a.size // ntr - 240) // 4
    assert ns == round(float(np.float32(time) / np.float32(dt))) // ndt
    for k in range(ntr):
        o = k * (240 + 4 * ns)
        # bytes 210-239 are header fields the reference never assigns (stack contents there)
        np.testing.assert_array_equal(a[o:o + 210], b[o:o + 210], err_msg=f"header of trace {k}")
        np.testing.assert_array_equal(a[o + 240:o + 240 + 4 * ns], b[o + 240:o + 240 + 4 * ns], err_msg=f"trace {k}")
    back = io.read_su(ours, ntr, ns)
    np.testing.assert_array_equal(back, sec[:, ndt - 1::ndt][:, :ns])


def _ref_outseis_fmt(path, fmt, sec, ri, rj, xs, ys, ndt, time, dt, dh, refx, refy):
    lib = ctypes.CDLL(O.REF_SO)
    sec = np.ascontiguousarray(sec, np.float32)
    ri = np.ascontiguousarray(ri, np.int32)
    rj = np.ascontiguousarray(rj, np.int32)
    f = ctypes.c_float
    assert lib.refh_outseis_fmt(path.encode(), fmt, O._fp(sec), sec.shape[0], sec.shape[1], O._ip(ri), O._ip(rj),
                                f(xs), f(ys), ndt, f(time), f(dt), f(dh), f(refx), f(refy)) == 0


@needs_ref
@pytest.mark.parametrize("fmt", [2, 3])
@pytest.mark.parametrize("ndt", [1, 3])
def test_ascii_and_binary_seismograms_match_outseis_glob(tmp_path, fmt, ndt):
    """SEIS_FORMAT 2 (one "%e" per line) and 3 (native floats), trace after trace,
    NDT-decimated: byte for byte the files of the reference's outseis_glob."""
    rng = np.random.default_rng(fmt + 10 * ndt)
    ntr, nt, dt, dh = 11, 200, 4e-4, 5.0
    time = np.float32(nt * dt)
    sec = (rng.standard_normal((ntr, nt)) * 10.0 ** rng.integers(-12, 3, (ntr, 1))).astype(np.float32)
    ri = np.arange(4, 4 + 3 * ntr, 3).astype(np.int32)
    rj = np.full(ntr, 5, np.int32)
    ours, ref = str(tmp_path / "ours"), str(tmp_path / "ref")
    io.write_seis(ours, fmt, sec, ndt, dt, time, dh, ri, rj, [0.0, 2.0, 1.0, 0.0], 312.5, 10.0)
    O.run_isolated(_ref_outseis_fmt, ref, fmt, sec, ri, rj, 312.5, 10.0, ndt, time, dt, dh, 2.0, 1.0)
    assert open(ours, "rb").read() == open(ref, "rb").read()


def test_model_file_roundtrip_and_short_file(tmp_path):
    a = np.random.default_rng(0).standard_normal((12, 7)).astype(np.float32)
    p = str(tmp_path / "m.vp")
    a.tofile(p)
    np.testing.assert_array_equal(io.read_model_file(p, 12, 7), a)
    with pytest.raises(io._lib.DeniseError) as e:
        io.read_model_file(p, 12, 8)
    assert e.value.code == io._lib.DN_EIO


def test_source_cell_rounding():
    # splitsrc: iround(x / DH) on the float quotient
    assert io.source_cell(12.5, 7.4999, 5.0) == (3, 1)
    assert io.source_cell(1497.5, 10.0, 5.0) == (300, 2)
