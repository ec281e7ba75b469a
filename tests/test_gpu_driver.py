"""The forward-modelling driver end to end: a parameter file, its model,
source and receiver files run by the reference's own program (oracle/_ref/denise,
CPU) and by this library (dn_forward_inp and the denise_b200 command, GPU); the
SU files must agree byte for byte: every trace's 210 header bytes the reference
assigns and every sample (the propagation is bit-exact)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracles as O
import inp_case
from denise_b200 import io

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "denise-black-edition_b200", "bin", "denise_b200")

CASES = {
    "elastic-fd8-fs": dict(),
    "visco-l3-fd4": dict(L=3, FDORDER=4),
    "elastic-all-components-ndt2": dict(SEISMO=4, NDT=2, FREE_SURF=0, FDORDER=6),
    "one-shot-all-sources": dict(RUN_MULTIPLE_SHOTS=0, nshots=2),
    "rotated-force-sources": dict(src_type=4),
    "spike-band-pass-quellart6": dict(QUELLART=6, FC_SPIKE_1=5.0, FC_SPIKE_2=40.0, ORDER_SPIKE=4),
    "spike-low-pass-quellart6": dict(QUELLART=6, FC_SPIKE_1=-5.0, FC_SPIKE_2=30.0, ORDER_SPIKE=5),
    "wavelet-file-quellart3": dict(QUELLART=3, SIGNAL_FILE="wavelet/sig", wavelet_files=True),
    "klauder-quellart7": dict(QUELLART=7, FC_SPIKE_1=7.0, FC_SPIKE_2=45.0),
    "seis-format-ascii": dict(SEIS_FORMAT=2, SEISMO=4, NDT=3),
    "seis-format-binary": dict(SEIS_FORMAT=3, SEISMO=1),
    "receivers-per-shot-readrec2": dict(READREC=2, per_shot_receivers=True),
}


def _su_equal(a_path, b_path, ntr):
    a = np.fromfile(a_path, np.uint8)
    b = np.fromfile(b_path, np.uint8)
    assert a.size == b.size, (a_path, a.size, b.size)
    per = a.size // ntr
    for k in range(ntr):
        o = k * per
        np.testing.assert_array_equal(a[o:o + 210], b[o:o + 210], err_msg=f"{a_path} header {k}")
        np.testing.assert_array_equal(a[o + 240:o + per], b[o + 240:o + per], err_msg=f"{a_path} trace {k}")


def _make(root, kw):
    kw = dict(kw)
    nshots = kw.pop("nshots", 3)
    styp = kw.pop("src_type", 1)
    wavelet_files = kw.pop("wavelet_files", False)
    per_shot = kw.pop("per_shot_receivers", False)
    inp = inp_case.write_case(root, nshots=nshots, **kw)
    if per_shot:   # READREC 2: "<REC_FILE>_shot_<n>.dat", a different line of receivers per shot
        lines = open(os.path.join(root, "receiver", "receivers.dat")).read().splitlines()
        for k in range(1, nshots + 1):
            with open(os.path.join(root, "receiver", f"receivers_shot_{k}.dat"), "w") as f:
                f.write("".join(ln + "\n" for ln in lines[k - 1: len(lines) - 2 * k]))
    if wavelet_files:   # QUELLART 3: "<SIGNAL_FILE>_shot_<n>.dat", one sample per line
        os.makedirs(os.path.join(root, "wavelet"), exist_ok=True)
        nt = io.inp_nt(io.read_inp(inp))
        for k in range(1, nshots + 1):
            rng = np.random.default_rng(100 + k)
            w = 1e3 * np.cumsum(rng.standard_normal(nt + 3)).astype(np.float32) / np.sqrt(nt)
            with open(os.path.join(root, "wavelet", f"sig_shot_{k}.dat"), "w") as f:
                f.write("".join(f"{v:.7e}\n" for v in w))
    if styp != 1:
        path = os.path.join(root, "source", "sources.dat")
        lines = open(path).read().splitlines()
        out = [lines[0]]
        for k, ln in enumerate(lines[1:]):
            c = ln.split("\t")
            c[6] = f"{30.0 + 20 * k:.2f}"
            c[7] = str(styp)
            out.append("\t".join(c))
        open(path, "w").write("\n".join(out) + "\n")
    return inp


@pytest.mark.skipif(not os.path.exists(O.REF_BIN), reason="reference program not built")
@pytest.mark.parametrize("name", list(CASES))
def test_driver_matches_reference_program(tmp_path, name):
    ref_dir, our_dir, cli_dir = (str(tmp_path / d) for d in ("ref", "ours", "cli"))
    for d in (ref_dir, our_dir, cli_dir):
        os.makedirs(d)
    _make(ref_dir, CASES[name])
    for d in (our_dir, cli_dir):
        shutil.rmtree(d)
        shutil.copytree(ref_dir, d)
    r = subprocess.run([O.REF_BIN, "case.inp"], cwd=ref_dir, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    cwd = os.getcwd()
    try:
        os.chdir(our_dir)
        io.forward_inp("case.inp", 0)
    finally:
        os.chdir(cwd)
    r = subprocess.run([CLI, "case.inp"], cwd=cli_dir, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    ref_files = sorted(f for f in os.listdir(os.path.join(ref_dir, "su")) if ".shot" in f)
    assert ref_files
    inp = io.read_inp(os.path.join(ref_dir, "case.inp"))
    for f in ref_files:
        shot = int(f.rsplit(".shot", 1)[1])
        rec = "receivers_shot_%d.dat" % shot if inp.readrec == 2 else "receivers.dat"
        ri, _ = io.read_receivers(os.path.join(ref_dir, "receiver", rec), inp.refrec, inp.dh)
        for d in (our_dir, cli_dir):
            if inp.seis_format == 1:
                _su_equal(os.path.join(d, "su", f), os.path.join(ref_dir, "su", f), len(ri))
            else:   # ASCII or raw floats: the whole file
                assert open(os.path.join(d, "su", f), "rb").read() == open(os.path.join(ref_dir, "su", f), "rb").read(), f
    ours = sorted(f for f in os.listdir(os.path.join(our_dir, "su")) if ".shot" in f)
    assert ours == ref_files
