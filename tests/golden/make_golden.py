"""Generates the golden fixtures of tests/golden/ by running the reference's own
code (oracle/_ref/libdenise_ref.so, built by oracle/Makefile from the
reference sources) on small seeded cases.

    python tests/golden/make_golden.py

Each case stores its inputs (so the fixtures do not depend on the model
generator) and the reference's outputs: setup arrays, sections, final
wavefields, per-shot correlation accumulators and gradients.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "denise-black-edition_b200"), os.path.join(ROOT, "tests")]

import numpy as np  # noqa: E402

import oracles as O  # noqa: E402
from denise_b200 import synth  # noqa: E402
from denise_b200.api import PsvParams  # noqa: E402

FL5 = (2.0, 8.0, 25.0, 1.0, 60.0)

CASES = {
    "elastic_fd8_fs": dict(L=0, fdorder=8, free_surf=1, styp=1),
    "visco_l3_fd8_fs": dict(L=3, fdorder=8, free_surf=1, styp=1),
    "elastic_fd4_force": dict(L=0, fdorder=4, free_surf=0, styp=3),
    "visco_l2_fd12_rot": dict(L=2, fdorder=12, free_surf=1, styp=4),
}


def case_inputs(L, fdorder, free_surf, styp, nx=64, ny=48, nt=300, seed=3):
    p = synth.c0_params(nx=nx, ny=ny, nt=nt, fw=10, L=L, fl=FL5[:L], ts=0.1, fdorder=fdorder,
                        free_surf=free_surf, dtinv=3, seismo=4, quelltypb=1, store_snapshots=1)
    vp, vs, rho = synth.base_model(nx, ny, p.dh, seed)
    qp, qs = synth.q_model(nx, ny, seed)
    sig = (synth.ricker_source(p, 40.0)[None, :] * 1e3).astype(np.float32)
    src = (np.array([nx // 2 - 2], np.int32), np.array([3], np.int32), sig, np.array([styp], np.int32),
           np.array([30.0], np.float32))
    nr = (nx - 10) // 4
    rec = (np.arange(5, 5 + 4 * nr, 4).astype(np.int32), np.full(nr, 4, np.int32))
    return p, (vp, vs, rho, qp, qs), src, rec


def residuals(p, syn):
    d = (syn - np.float32(0.7) * syn).astype(np.float32)
    d[:, 0] = 0.0
    out = np.zeros_like(d)
    acc = np.zeros(d.shape[0], np.float32)
    for t in range(p.nt):
        acc = (acc + np.float32(p.dt) * d[:, t]).astype(np.float32)
        out[:, p.nt - 1 - t] = acc
    return out


def run_reference(p, model, src, rec):
    r = O.Reference(p, model, src, rec, mode_global=1)
    out = {"hc": r.hc(), "pml": r.pml(), "rip": r.mat(0), "rjp": r.mat(1), "uipjp": r.mat(2)}
    if p.L:
        for k, n in enumerate(("fipjp", "f", "g")):
            out[n] = r.mat(3 + k)
        out["dip"] = np.stack([r.mat(100 + l) for l in range(1, p.L + 1)])
        out["d"] = np.stack([r.mat(200 + l) for l in range(1, p.L + 1)])
        out["e"] = np.stack([r.mat(300 + l) for l in range(1, p.L + 1)])
        out["visc_vectors"] = r.visc_vectors()
    r.run(0)
    for c in range(5):
        out[f"sec{c}"] = r.sections(c)
    for f in range(7):
        out[f"field{f}"] = r.field(f)
    rvx, rvy = residuals(p, out["sec0"]), residuals(p, out["sec1"])
    out["res_vx"], out["res_vy"] = rvx, rvy
    r.set_residuals(rvx, rvy, None)
    r.run(1)
    for f in (7, 8, 9):
        out[f"field{f}"] = r.field(f)
    out["gvp"], out["gvs"], out["grho"] = r.ass_grad()
    wav = {}
    for qa in (1, 2, 4, 5, 6):
        wav[f"wavelet{qa}"] = np.zeros(p.nt, np.float32)
        r.lib.refh_wavelet(qa, 0, O.ctypes.c_float(0.0), O.ctypes.c_float(25.0), O.ctypes.c_float(1.5),
                           wav[f"wavelet{qa}"].ctypes.data_as(O._f))
    out.update(wav)
    return out


def main():
    if not O.reference_available():
        sys.exit("build the reference oracle first: make -C oracle reference")
    for name, kw in CASES.items():
        p, model, src, rec = case_inputs(**kw)
        out = O.run_isolated(run_reference, p, model, src, rec)
        meta = {k: (list(v) if isinstance(v, tuple) else v) for k, v in p.__dict__.items()}
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), params=json.dumps(meta),
                            vp=model[0], vs=model[1], rho=model[2], qp=model[3], qs=model[4],
                            src_i=src[0], src_j=src[1], signals=src[2], src_type=src[3], src_azi=src[4],
                            rec_i=rec[0], rec_j=rec[1], **out)
        print(name, "written")


def load(name):
    z = np.load(os.path.join(HERE, f"{name}.npz"))
    meta = json.loads(str(z["params"]))
    meta["fl"] = tuple(meta["fl"])
    p = PsvParams(**meta)
    model = (z["vp"], z["vs"], z["rho"], z["qp"], z["qs"])
    src = (z["src_i"], z["src_j"], z["signals"], z["src_type"], z["src_azi"])
    rec = (z["rec_i"], z["rec_j"])
    return p, model, src, rec, z


if __name__ == "__main__":
    main()
