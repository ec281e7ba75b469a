"""Benchmark of the B200 P-SV propagator on the batched viscoelastic workload.

Workload (one "step"): 64 viscoelastic shots (L = 3, FDORDER 8, CPML 20,
free surface), each on its own 2000 x 600 model (DH 5 m) with 400 receivers,
run through the whole time loop of NT = 6000 steps (DT 0.4 ms) as one batched,
graph-replayed launch per operation.  Metric: Mcell-updates/s = shots x NX x
NZ x NT / time.  Inputs (~15 GB resident) are larger than L2, so no flush is
needed between timed steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank runs its own 64-shot batch (shots are independent:
weak scaling, no collective on the data path); rank 0 prints one JSON line.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "denise-black-edition_b200")
for _p in (PKG, os.path.join(ROOT, "tests")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "Elastic Mcell-updates/s, HBM % peak; batched shots/s vs plain; p50/p99 latency"
UNIT = "Mcell-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--shots", type=int, default=64)
    ap.add_argument("--nt", type=int, default=6000)
    ap.add_argument("--nx", type=int, default=2000)
    ap.add_argument("--ny", type=int, default=600)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--plain-shots", type=int, default=4)
    ap.add_argument("--cpu-sample-nt", type=int, default=60)
    ap.add_argument("--serve-requests", type=int, default=32,
                    help="requests of the serving workload run after the batch measurement (0: skip)")
    ap.add_argument("--serve-scale", type=float, default=1.0, help="shrinks NX, NZ and NT of served requests")
    ap.add_argument("--gradient-shots", type=int, default=32,
                    help="shots of the FWI-gradient measurement (1700x500, NT 4000, FP16 snapshots; 0: skip)")
    ap.add_argument("--fwi-large-shots", type=int, default=0,
                    help="shots of a sample of the 8000x2000, NT 12000 FWI iteration (0: skip)")
    ap.add_argument("--elastic-nt", type=int, default=1000,
                    help="NT of the elastic batch measured beside the viscoelastic one (0: skip)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# reference CPU path (oracle/_ref: the reference's own code, or the C port)
# ---------------------------------------------------------------------------
def _modelgen():
    """denise_b200/modelgen.py loaded by file path: the workload's numpy model and
    acquisition generators without importing the package (which loads the CUDA
    library), so the reference arm runs nothing but the reference's own code."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("dn_modelgen", os.path.join(PKG, "denise_b200", "modelgen.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _cpu_worker(args):
    """One process: one shot of the workload for `nt_sample` steps on the reference's code."""
    kind, k, nx, ny, nt_sample, seed = args
    import oracles as O

    mg = _modelgen()
    p = mg.c1_reference_params(nx=nx, ny=ny, nt=nt_sample)
    model = mg.base_model(nx, ny, p.dh, seed) + mg.q_model(nx, ny, seed)
    (si, sj), rec = mg.c1_acquisition(nx, ny, p.dh, k % 64)
    sig = mg.ricker(nt_sample, p.dt, 8.0)[None, :]
    src = (si, sj, sig, np.ones(1, np.int32), np.zeros(1, np.float32))
    if kind == "reference":
        r = O.Reference(p, model, src, rec, mode_global=0)
        t0 = time.perf_counter()
        r.run(0)
        return time.perf_counter() - t0
    r = O.Restatement(p, model, src, rec, "f")
    t0 = time.perf_counter()
    r.forward(store=False)
    return time.perf_counter() - t0


def cpu_sample(nx, ny, nt_sample, nproc=None):
    """Runs nproc concurrent single-rank shots on the host cores; returns (Mcell/s, cores, kind, secs)."""
    import multiprocessing as mp

    import oracles as O

    kind = "reference" if O.reference_available() else "port"
    nproc = nproc or min(os.cpu_count() or 1, 64)
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(nproc) as pool:
        times = pool.map(_cpu_worker, [(kind, k, nx, ny, nt_sample, 1000 + k) for k in range(nproc)])
    wall = time.perf_counter() - t0
    cells = nproc * nx * ny * nt_sample
    rate = cells / max(times) / 1e6
    return rate, nproc, kind, max(times), wall


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[3 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def traffic_per_cell(kernel):
    """DRAM bytes per cell of one launch from the committed ncu capture (profiles/traffic.json)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return float(json.load(f)[kernel]["dram_bytes_per_cell"])
    except Exception:
        return None


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def build_inputs(p, nshots, shot_offset):
    from denise_b200 import synth

    return [synth.c1_shot(p, k % 64, nshots=64, seed=1 + k + shot_offset) for k in range(nshots)]


def create_batch(p, inputs, device):
    from concurrent.futures import ThreadPoolExecutor

    import denise_b200 as dn

    def mk(inp):
        model, src, rec = inp
        m = dn.Model(p, *model, device=device)
        s = dn.Shot(m, src[0], src[1], src[2], rec[0], rec[1])
        return m, s

    with ThreadPoolExecutor(max_workers=min(16, len(inputs))) as ex:
        return list(ex.map(mk, inputs))


def workload_config(a, p, world):
    return {"workload": f"batched viscoelastic forward: {a.shots} shots x {p.nx}x{p.ny} grid, NT={p.nt}, "
                        f"L=3, FDORDER 8, FW 20, free surface, 400 receivers/shot",
            "shots_per_gpu": a.shots, "nx": p.nx, "nz": p.ny, "nt": p.nt, "fdorder": p.fdorder, "L": p.L,
            "arith": "exact (bit-identical to the reference)",
            "l2_flush": "inputs larger than L2 (resident state ~15 GB)",
            "parallelism": f"shots-dp{world}"}


def run_ours(a, rank, world, local_rank):
    import denise_b200 as dn
    from denise_b200 import synth

    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist_mod
        from datetime import timedelta

        torch.cuda.set_device(local_rank)
        dist_mod.init_process_group("nccl", timeout=timedelta(seconds=600))
        dist = dist_mod
    device = local_rank
    p = synth.c1_params(nx=a.nx, ny=a.ny, nt=a.nt)
    cells_step = a.shots * p.nx * p.ny * p.nt

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        rate, cores, kind, secs, wall = cpu_sample(p.nx, p.ny, a.cpu_sample_nt)
        cpu = {"value": round(rate, 3), "unit": UNIT, "cores": cores, "kind": kind,
               "sample": f"{cores} concurrent single-rank shots of the {p.nx}x{p.ny} L=3 FDORDER 8 workload, "
                         f"{a.cpu_sample_nt} time steps each ({secs:.1f} s)"}

    inputs = build_inputs(p, a.shots, rank * a.shots)
    pairs = create_batch(p, inputs, device)
    shots = [s for _, s in pairs]

    def barrier():
        if dist is not None:
            dist.barrier()

    import torch

    for _ in range(a.warmup):
        dn.run(shots)
    torch.cuda.synchronize(device)
    barrier()
    with ClockSampler(device) as clk:
        t0 = time.perf_counter()
        dev_ms = 0.0
        launches = 0
        for _ in range(a.steps):
            dn.run(shots)
            ms, nl = dn.last_run_stats()
            dev_ms += ms
            launches += nl
        torch.cuda.synchronize(device)
        wall = time.perf_counter() - t0
    barrier()
    t_dev = dev_ms / 1e3
    if dist is not None:
        tt = torch.tensor([t_dev], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_dev = float(tt.item())
    value = cells_step * a.steps * world / t_dev / 1e6
    ms_step = t_dev / a.steps * 1e3

    result = None
    if rank == 0:
        # per-kernel times of the same batch (direct launches with events between kernels)
        prof = dn.api.profile_steps(shots, dn.MODE_FORWARD, nsteps=20)
        cells = a.shots * p.nx * p.ny
        peak, peak_kind = measured_peak()
        s_bytes = (14 + 6 * p.L) * 4 * cells       # stress kernel algorithmic bytes per launch
        v_bytes = 9 * 4 * cells
        achieved = s_bytes / (prof["update_s"] * 1e-3) / 1e9
        step_bytes = (23 + 6 * p.L) * 4 * cells
        step_ms = sum(prof.values())
        tpc = traffic_per_cell("k_update_s_vi<4,3>")
        roof = {"bound": "hbm", "kernel": "k_update_s_vi<4,3,true> (viscoelastic stress update)",
                "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "peak_kind": peak_kind + " (burst copy bandwidth)",
                "traffic": round(tpc * cells) if tpc else None,
                "traffic_note": "ncu dram bytes per cell of a 4-shot capture, scaled to this launch's cells",
                "algorithmic_bytes_per_launch": s_bytes,
                "v_kernel_gbs": round(v_bytes / (prof["update_v"] * 1e-3) / 1e9, 1),
                "whole_step_gbs_direct": round(step_bytes / (step_ms * 1e-3) / 1e9, 1),
                "kernel_ms": {k: round(v, 4) for k, v in prof.items()}}
        # plain (one shot at a time, direct launches) on a subset
        plain_shots = shots[: max(1, min(a.plain_shots, len(shots)))]
        torch.cuda.synchronize(device)
        tp = 0.0
        for s in plain_shots:
            dn.run_plain(s)
            tp += dn.last_run_stats()[0] / 1e3
        plain_sps = len(plain_shots) / tp
        batched_sps = a.shots * a.steps / t_dev
        elastic = None
        if a.elastic_nt > 0:
            elastic = run_elastic(a, inputs, device, peak)
        gradient = None
        if a.gradient_shots > 0:
            for m_, s_ in pairs:       # the gradient batches need the HBM
                s_.close()
                m_.close()
            gradient = run_gradient(a, device)
        fwi_large = None
        if a.fwi_large_shots > 0:
            for m_, s_ in pairs:
                s_.close()
                m_.close()
            fwi_large = run_fwi_large(a, device)
        serving = None
        if a.serve_requests > 0:
            for m_, s_ in pairs:       # free the batch's HBM for the served requests
                s_.close()
                m_.close()
            serving = run_serving(a, device, value)
        e2e = None
        if not a.no_e2e:
            e2e = run_e2e(p, inputs, device, cells_step)
        result = {
            "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(ms_step, 2), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded model family, see denise_b200/synth.py)",
            "config": workload_config(a, p, world),
            "shots_per_s": {"batched": round(batched_sps, 3), "plain": round(plain_sps, 3),
                            "speedup": round(batched_sps / plain_sps, 3),
                            "plain_sample_shots": len(plain_shots)},
            "roofline": roof,
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "wall_s_timed": round(wall, 3),
        }
        if elastic:
            result["elastic"] = elastic
        if serving:
            result["serving"] = serving
        if gradient:
            result["gradient"] = gradient
        if fwi_large:
            result["fwi_large"] = fwi_large
        if e2e:
            result["e2e"] = e2e
        if cpu:
            result["cpu_baseline"] = cpu
    for m, s in pairs:
        s.close()
        m.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return result


def run_elastic(a, inputs, device, peak):
    """The same shots with the elastic propagator (vp, vs, rho of each model, L = 0) at NT = a.elastic_nt:
    device time of the batched run, and the elastic step's per-kernel roofline."""
    import denise_b200 as dn
    import torch
    from denise_b200 import synth

    p = synth.c1_params(nx=a.nx, ny=a.ny, nt=a.elastic_nt, L=0, fl=())
    sig = synth.ricker_source(p, 8.0)[None, :]
    pairs = []
    for model, src, rec in inputs:
        m = dn.Model(p, *model[:3], device=device)
        pairs.append((m, dn.Shot(m, src[0], src[1], sig, rec[0], rec[1])))
    shots = [s for _, s in pairs]
    dn.run(shots)
    torch.cuda.synchronize(device)
    ms = 0.0
    for _ in range(2):
        dn.run(shots)
        ms += dn.last_run_stats()[0]
    ms /= 2
    cells = len(shots) * p.nx * p.ny
    prof = dn.api.profile_steps(shots, dn.MODE_FORWARD, nsteps=20)
    step_ms = sum(prof.values())
    out = {"value": round(cells * p.nt / (ms * 1e-3) / 1e6, 1), "unit": UNIT, "shots": len(shots), "nt": p.nt,
           "ms_per_run": round(ms, 2),
           "v_kernel_gbs": round(36 * cells / (prof["update_v"] * 1e-3) / 1e9, 1),
           "s_kernel_gbs": round(44 * cells / (prof["update_s"] * 1e-3) / 1e9, 1),
           "whole_step_gbs_direct": round(80 * cells / (step_ms * 1e-3) / 1e9, 1)}
    out["whole_step_frac"] = round(out["whole_step_gbs_direct"] / peak, 4)
    for m, s in pairs:
        s.close()
        m.close()
    return out


def run_gradient(a, device):
    """FWI gradient (forward with snapshots + adjoint) of the 1700 x 500 elastic workload:
    true model = the seeded family (seed 2), starting model = it smoothed with sigma 25
    cells, observed data synthesised on the GPU from the true model; FP16 snapshots
    every 2 steps; shots streamed through HBM in batches that fit."""
    import ctypes

    import denise_b200 as dn
    import torch
    from denise_b200 import synth

    import oracles as O

    p = synth.c2_params(snap_precision=dn.SNAP_F16)
    n = a.gradient_shots
    vpt, vst, rhot = synth.base_model(p.nx, p.ny, p.dh, 2)
    start = tuple(synth.smoothed(x, 25.0) for x in (vpt, vst, rhot))
    xmax = (p.nx - 1) * p.dh
    sig = synth.ricker_source(p, 8.0)[None, :]
    ri, rj = synth.receivers_line(100.0, xmax - 100.0, 400, 20.0, p.dh)
    shots = [(np.array([synth.grid_index(200.0 + (xmax - 400.0) * k / max(n - 1, 1), p.dh)], np.int32),
              np.array([max(synth.grid_index(10.0, p.dh), 1)], np.int32), sig, ri, rj) for k in range(n)]
    # observed data from the true model (batched forward, no snapshots)
    mt = dn.Model(p.replace(store_snapshots=0), vpt, vst, rhot, device=device)
    st_ = [dn.Shot(mt, *sh) for sh in shots]
    dn.run(st_)
    obs = [(s.sections(dn.SEC_VX), s.sections(dn.SEC_VY)) for s in st_]
    for s in st_:
        s.close()
    mt.close()
    fp = ctypes.c_size_t()
    pc = p.to_c()
    dn._lib.check(dn._lib.lib.dn_shot_footprint(ctypes.byref(pc), len(ri), 1, ctypes.byref(fp)))
    free, total = dn.device_memory(device)
    # as many shots per batch as 90 % of the free HBM holds, spread evenly over the
    # batches (32 shots: 4 x 8 rather than 4 x 7 + 4; larger batches run faster per shot)
    most = max(1, min(n, int(0.9 * free / fp.value)))
    nbatch = -(-n // most)
    batch = -(-n // nbatch)

    def grad(params, idx):
        m = dn.Model(params, *start, device=device)
        L2, dev_ms = 0.0, 0.0
        for b0 in range(0, len(idx), batch):
            ss = [dn.Shot(m, *shots[k]) for k in idx[b0:b0 + batch]]
            dn.run(ss, dn.MODE_FORWARD)
            dev_ms += dn.last_run_stats()[0]
            for s, k in zip(ss, idx[b0:b0 + batch]):
                L2 += s.residual(obs[k][0], dn.SEC_VX) + s.residual(obs[k][1], dn.SEC_VY)
            dn.run(ss, dn.MODE_ADJOINT)
            dev_ms += dn.last_run_stats()[0]
            for s in ss:
                s.accumulate_gradient()
                s.close()
        g = m.gradient()
        m.close()
        return g, L2, dev_ms

    grad(p, [0])                                   # warm-up (graphs, module load)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    g16, L2, dev_ms = grad(p, list(range(n)))
    torch.cuda.synchronize(device)
    wall = time.perf_counter() - t0
    cells = n * p.nx * p.ny * p.nt * 2
    g32, _, _ = grad(p.replace(snap_precision=dn.SNAP_F32), [0, n // 2])
    g16s, _, _ = grad(p, [0, n // 2])
    err = max(O.rel_l2(x, y) for x, y in zip(g16s, g32))
    return {"workload": f"FWI gradient, elastic {p.nx}x{p.ny}, DH {p.dh} m, DT {p.dt} s, NT {p.nt}, FDORDER 8, "
                        f"{n} shots x 400 receivers, FP16 snapshots every DTINV={p.dtinv} steps, "
                        "starting model smoothed sigma 25 cells, observed data synthesised on the GPU",
            "shots": n, "batch_shots": batch, "seconds": round(wall, 2),
            "device_ms": round(dev_ms, 1), "shots_per_s": round(n / wall, 3),
            "mcell_updates_per_s": round(cells / wall / 1e6, 1),
            "misfit": L2, "fp16_vs_fp32_gradient_rel_l2": float(err)}


def run_fwi_large(a, device):
    """A sample of the large FWI iteration: elastic 8000 x 2000, DH 2.5 m, DT 0.2 ms
    (0.25 ms breaks the CFL limit of this model), NT 12000, FDORDER 8, shots of the
    96-shot line with 1600 receivers; true model = the seeded family (seed 4) plus a
    5500 m/s ellipse, starting model smoothed with sigma 25 cells; one FWI iteration
    with FP16 snapshots every 4 steps and checkpointed adjoints (segments of 400
    steps), the FP64 L-BFGS direction, the parabolic step search and the update."""
    import denise_b200 as dn
    from denise_b200 import fwi, synth
    from denise_b200.api import PsvParams

    n = a.fwi_large_shots
    p = PsvParams(nx=8000, ny=2000, dh=2.5, dt=2e-4, nt=12000, fdorder=8, fw=20, free_surf=1, ts=0.125,
                  store_snapshots=1, dtinv=4, snap_precision=dn.SNAP_F16, ckpt_steps=400)
    t0 = time.perf_counter()
    vp, vs, rho = synth.base_model(p.nx, p.ny, p.dh, 4)
    true = synth.add_ellipse(vp, vs, rho, p.dh, 4, v=5500.0)
    start = tuple(synth.smoothed(x, 25.0) for x in true)
    xmax = (p.nx - 1) * p.dh
    sig = synth.ricker_source(p, 8.0)[None, :]
    ri, rj = synth.receivers_line(100.0, xmax - 100.0, 1600, 20.0, p.dh)
    picks = np.linspace(0, 95, n).round().astype(int)
    shots = [(np.array([synth.grid_index(200.0 + (xmax - 400.0) * k / 95.0, p.dh)], np.int32),
              np.array([max(synth.grid_index(10.0, p.dh), 1)], np.int32), sig, ri, rj) for k in picks]
    t1 = time.perf_counter()
    po = p.replace(store_snapshots=0, ckpt_steps=0)
    mt = dn.Model(po, *true, device=device)
    st_ = [dn.Shot(mt, *sh) for sh in shots]
    dn.run(st_)
    fwd_ms = dn.last_run_stats()[0]
    obs = [(s.sections(dn.SEC_VX), s.sections(dn.SEC_VY)) for s in st_]
    for s in st_:
        s.close()
    mt.close()
    t2 = time.perf_counter()
    lim = (1000.0, 6500.0, 500.0, 4000.0, 1000.0, 3500.0)
    f = fwi.FWI(p, start, shots, obs, lim, device=device, nlbfgs=5, eps_scale=0.01)
    L2 = f.iterate(1)
    h = f.history[-1]
    L2_new = f.misfit((f.vp, f.vs, f.rho))
    f.close()
    t3 = time.perf_counter()
    cells = p.nx * p.ny * p.nt
    per_shot_grad = h["gradient_s"] / n
    per_shot_fwd = fwd_ms / 1e3 / n
    return {"workload": "FWI iteration sample: elastic 8000x2000, DH 2.5 m, DT 0.2 ms, NT 12000, FDORDER 8, "
                        f"{n} of 96 shots x 1600 receivers, FP16 snapshots every 4 steps, checkpointed adjoint "
                        "(400-step segments), FP64 L-BFGS, parabolic step search",
            "shots": n, "setup_s": round(t1 - t0, 1), "observed_data_s": round(t2 - t1, 1),
            "forward_device_s_per_shot": round(per_shot_fwd, 2),
            "forward_mcell_updates_per_s": round(cells / per_shot_fwd / 1e6, 1),
            "gradient_s": round(h["gradient_s"], 1), "gradient_s_per_shot": round(per_shot_grad, 2),
            "optimizer_s": round(h["optimizer_s"], 3), "step_search_s": round(h["step_search_s"], 1),
            "test_models": h["test_models"], "step_found": h["found"], "eps": h["eps"],
            "misfit_before": L2, "misfit_after": L2_new,
            "iteration_s": round(t3 - t2, 1),
            "iteration_96_shots_estimate_s": round(96 * per_shot_grad + h["test_models"] * 96 * per_shot_fwd, 0)}


def run_serving(a, device, mcells_per_s):
    """The serving workload: requests arrive as a Poisson process at 1.2x the
    capacity implied by the batched throughput just measured; the server admits
    them by HBM footprint into its run queues.  Latency = scheduled arrival ->
    result on the host."""
    from denise_b200 import serve, synth

    reqs = synth.serve_requests(a.serve_requests, seed=3, scale=a.serve_scale)
    work = []
    for kind, p, model, shots, obs in reqs:
        w = p.nx * p.ny * p.nt * len(shots)
        work.append(2 * w if kind == "gradient" else w)
    rate = 1.2 * mcells_per_s * 1e6 / float(np.mean(work))      # requests per second
    rng = np.random.default_rng(3)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
    srv = serve.Server(device=device, chunk=50)
    t0 = time.perf_counter()
    i = 0
    while i < len(reqs) or not srv.idle():
        now = time.perf_counter() - t0
        while i < len(reqs) and arrivals[i] <= now:
            kind, p, model, shots, obs = reqs[i]
            srv.submit(serve.Request(kind, p, model, shots, obs, rid=i), now=t0 + arrivals[i])
            i += 1
        if srv.idle():
            time.sleep(max(0.0, min(0.05, arrivals[i] - (time.perf_counter() - t0))))
            continue
        srv.step()
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    bad = sum(1 for r in srv.results if r.status != 0)
    return {"requests": len(reqs), "failed": bad, "p50_latency_s": round(st["p50_s"], 3),
            "p99_latency_s": round(st["p99_s"], 3), "shots_per_s": round(st["shots_done_total"] / wall, 3),
            "mcell_updates_per_s": round(sum(work) / wall / 1e6, 1), "wall_s": round(wall, 2),
            "arrival_rate_per_s": round(rate, 3), "max_running_shots": st["max_running_shots"],
            "joins_while_running": st["joins_while_running"],
            "workload": "seeded serving mix: 70% elastic forward, 20% visco L=3 forward, 10% elastic FWI gradient "
                        "(FP16 snapshots); NX 300-3000, NZ 150-1000, NT 2000-8000 (x scale "
                        f"{a.serve_scale}), FDORDER 4/8/12, 1-4 shots, 50-500 receivers; Poisson arrivals at 1.2x "
                        "the batched capacity"}


def run_e2e(p, inputs, device, cells_step):
    """One step through the public API with host buffers: models/shots created from host arrays
    (host set-up + H2D), the batched run, sections read back (D2H), objects freed."""
    import denise_b200 as dn
    import torch

    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    pairs = create_batch(p, inputs, device)
    shots = [s for _, s in pairs]
    dn.run(shots)
    secs = [(s.sections(dn.SEC_VX), s.sections(dn.SEC_VY)) for s in shots]
    for m, s in pairs:
        s.close()
        m.close()
    torch.cuda.synchronize(device)
    t = time.perf_counter() - t0
    h2d = sum(5 * m[0].size * 4 + src[2].nbytes + 8 * len(rec[0]) + 8 for m, src, rec in inputs)
    d2h = sum(a.nbytes + b.nbytes for a, b in secs)
    return {"value": round(cells_step / t / 1e6, 1), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "steps": 1, "seconds": round(t, 3)}


def run_reference(a, rank, world):
    if rank != 0:
        return None
    p = _modelgen().c1_reference_params(nx=a.nx, ny=a.ny, nt=a.nt)
    for _ in range(a.warmup):
        cpu_sample(p.nx, p.ny, max(2, a.cpu_sample_nt // 6))
    rates, secs = [], []
    for _ in range(a.steps):
        rate, cores, kind, sec, wall = cpu_sample(p.nx, p.ny, a.cpu_sample_nt)
        rates.append(rate)
        secs.append(sec)
    value = float(np.median(rates))
    ms = float(np.median(secs)) * 1e3
    sample = (f"{cores} concurrent single-rank shots of the {p.nx}x{p.ny} L=3 FDORDER 8 workload, "
              f"{a.cpu_sample_nt} time steps each per step")
    return {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(ms, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": dict(workload_config(a, p, world), parallelism="host processes",
                           sample="bounded: one single-rank process per host core, each on its own shot of this "
                                  f"workload for {a.cpu_sample_nt} time steps"),
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    a = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if a.impl == "reference":
        res = run_reference(a, rank, world)
    else:
        res = run_ours(a, rank, world, local_rank)
    if rank == 0 and res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
