"""Benchmark of the B200 P-SV propagator on the batched viscoelastic workload.

Workload (one "step"): 64 viscoelastic shots (L = 3, FDORDER 8, CPML 20,
free surface), each on its own 2000 x 600 model (DH 5 m) with 400 receivers,
run through the whole time loop of NT = 6000 steps (DT 0.4 ms) as one batched,
graph-replayed launch per operation.  Metric: Mcell-updates/s = shots x NX x
NZ x NT / time.  Inputs (~15 GB resident) are larger than L2, so no flush is
needed between timed steps.

Beside the headline the JSON line carries the other workloads: `c0` (the
plain single-shot elastic forward, 600 x 300, NT 5000: batched and plain
paths, end to end, the reference's own full run on one core and a bitwise
comparison with it), `elastic` (the 2000 x 600 grid of 64 shots, elastic, NT
6000), `gradient` (the 1700 x 500, NT 4000, 32-shot FWI gradient with FP16
snapshots, and on one of its shots the errors of the FP32 gradient against the
reference's and of the FP16 gradient against the FP64 restatement, both timed
on the host as CPU baselines), `serving` (the mixed request stream with its
load calibrated to the measured capacity of the mix) and `fwi_large` (shots of
the 8000 x 2000, NT 12000 FWI iteration with batched checkpointed adjoints).

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
    ap.add_argument("--serve-requests", type=int, default=500,
                    help="requests of the serving workload run after the batch measurement (0: skip)")
    ap.add_argument("--serve-calibration", type=int, default=48,
                    help="requests of the closed-loop run that measures the serving capacity of the mix")
    ap.add_argument("--serve-scale", type=float, default=1.0, help="shrinks NX, NZ and NT of served requests")
    ap.add_argument("--gradient-shots", type=int, default=32,
                    help="shots of the FWI-gradient measurement (1700x500, NT 4000, FP16 snapshots; 0: skip)")
    ap.add_argument("--fwi-large-shots", type=int, default=4,
                    help="shots of a sample of the 8000x2000, NT 12000 FWI iteration (0: skip)")
    ap.add_argument("--elastic-nt", type=int, default=6000,
                    help="NT of the elastic batch measured beside the viscoelastic one (0: skip)")
    ap.add_argument("--no-c0", action="store_true", help="skip the plain single-shot elastic workload")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the host runs of the reference and the FP64 restatement beside the GPU work")
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


def kernel_choice(p):
    """The tile and stencil-kernel variant the library's rules give this workload."""
    try:
        from denise_b200 import tune

        bx, zch, v = tune.choice_for(p)
        return {"tile": f"{bx}x{zch}", "variant": {0: "paired-column FP32x2", 1: "one-column",
                                                   2: "paired, pipelined velocity",
                                                   3: "fused elastic step"}.get(v, str(v)),
                "rule": "the library's default (tile_choice), which the table measured by denise_b200.tune "
                        "(denise_b200/tiles_b200.json) confirms"}
    except Exception:
        return None


def workload_config(a, p, world, ours=True):
    return {"workload": f"batched viscoelastic forward: {a.shots} shots x {p.nx}x{p.ny} grid, NT={p.nt}, "
                        f"L=3, FDORDER 8, FW 20, free surface, 400 receivers/shot",
            "shots_per_gpu": a.shots, "nx": p.nx, "nz": p.ny, "nt": p.nt, "fdorder": p.fdorder, "L": p.L,
            "arith": "exact (bit-identical to the reference)", "kernels": kernel_choice(p) if ours else None,
            "l2_flush": "inputs larger than L2 (resident state ~15 GB)",
            "parallelism": f"shots-dp{world}"}


class HostJobs:
    """CPU runs beside the GPU work, in spawned processes started before the
    timed regions need the host: the reference's own full C0 run (the C0 CPU
    baseline and its bitwise comparison) and, on one shot of the FWI-gradient
    workload, the reference's gradient (grad_obj_psv's shot loop: forward with
    snapshots, calc_res, adjoint, ass_gradPSV) and then the FP64 restatement's
    gradient with the GPU's adjoint sources.  The C2 runs hold 34 GB (reference)
    and 68 GB (FP64) of host snapshot arrays one after the other; they are
    skipped when the host has less memory free."""

    def __init__(self):
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor

        self.ex = ProcessPoolExecutor(max_workers=2, mp_context=mp.get_context("spawn"))
        self.futs = {}
        self.notes = {}
        self._chain = None

    def c0(self, p, model, src, rec):
        import config_cases as CC

        self.futs["c0"] = self.ex.submit(CC.ref_forward, p, model, src, rec)

    def c2(self, p, start, shot, obs, residual):
        import config_cases as CC

        need_ref, need_64 = CC.snapshot_bytes(p, 4), CC.snapshot_bytes(p, 8)
        avail = CC.available_memory()
        if avail < 1.3 * need_ref:
            self.notes["c2"] = f"skipped: {avail / 1e9:.0f} GB of host memory free"
            return
        self.futs["c2_ref"] = self.ex.submit(CC.ref_gradient_shot, p, start, shot, obs[0], obs[1])

        def chain():
            try:
                self.futs["c2_ref"].result()
            except Exception:
                return
            if CC.available_memory() < 1.3 * need_64:
                self.notes["c2_fp64"] = "skipped: host memory"
                return
            self.futs["c2_fp64"] = self.ex.submit(CC.fp64_gradient, p, start, [shot], [residual], 8)

        self._chain = threading.Thread(target=chain, daemon=True)
        self._chain.start()

    def result(self, key, timeout=3600):
        if key == "c2_fp64" and self._chain is not None:
            self._chain.join(timeout)
        f = self.futs.get(key)
        if f is None:
            return None
        try:
            return f.result(timeout=timeout)
        except Exception as e:      # a failed host run is reported, not fatal
            self.notes[key] = f"failed: {type(e).__name__}: {e}"[:300]
            return None

    def close(self):
        self.ex.shutdown(wait=True, cancel_futures=True)


def c2_parity_inputs(device):
    """Shot 0 of the FWI-gradient workload: observed data of the true model, and the
    GPU's FP32 and FP16-snapshot gradients with the L2 adjoint sources of its
    own FP32 forward run (calc_res, oracle/residual_oracle.py, equal to the device
    residual bit for bit)."""
    import denise_b200 as dn

    import config_cases as CC
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import residual_oracle as ro

    p, true, start, shots = CC.c2_case()
    sh = shots[0]
    mt = dn.Model(p.replace(store_snapshots=0), *true, device=device)
    s = dn.Shot(mt, *sh)
    dn.run([s])
    obs = (s.sections(dn.SEC_VX), s.sections(dn.SEC_VY))
    s.close()
    mt.close()
    grads, res = {}, None
    for prec in (dn.SNAP_F32, dn.SNAP_F16):
        m = dn.Model(p.replace(snap_precision=prec), *start, device=device)
        s = dn.Shot(m, *sh)
        dn.run([s], dn.MODE_FORWARD)
        if res is None:
            res = (ro.calc_res(obs[0], s.sections(dn.SEC_VX), p.dt)[0], ro.calc_res(obs[1], s.sections(dn.SEC_VY), p.dt)[0])
        s.set_residuals(res[0], res[1], None)
        dn.run([s], dn.MODE_ADJOINT)
        s.accumulate_gradient()
        grads[prec] = m.gradient()
        s.close()
        m.close()
    return p, start, sh, obs, res, grads


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
    side = rank == 0 and world == 1      # the side workloads and host baselines: one GPU, rank 0

    cpu = None
    if side and not a.no_cpu:
        rate, cores, kind, secs, wall = cpu_sample(p.nx, p.ny, a.cpu_sample_nt)
        cpu = {"value": round(rate, 3), "unit": UNIT, "cores": cores, "kind": kind,
               "sample": f"{cores} concurrent single-rank shots of the {p.nx}x{p.ny} L=3 FDORDER 8 workload, "
                         f"{a.cpu_sample_nt} time steps each ({secs:.1f} s)"}

    jobs, c0case, c2in = None, None, None
    if side and not a.no_parity:
        jobs = HostJobs()
        if not a.no_c0:
            c0case = synth.c0_case(seed=0)
            jobs.c0(*c0case)
        if a.gradient_shots > 0:
            c2in = c2_parity_inputs(device)
            jobs.c2(c2in[0], c2in[1], c2in[2], c2in[3], c2in[4])

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
        e2e = None
        if not a.no_e2e:
            e2e = run_e2e(p, inputs, device, cells_step)
        blocks = {}
        if side:
            if not a.no_c0:
                blocks["c0"] = run_c0(a, device, peak, c0case, jobs)
            if a.elastic_nt > 0:
                blocks["elastic"] = run_elastic(a, inputs, device, peak)
            for m_, s_ in pairs:       # the remaining workloads need the HBM
                s_.close()
                m_.close()
            pairs = []
            if a.gradient_shots > 0:
                blocks["gradient"] = run_gradient(a, device, c2in, jobs)
            if a.fwi_large_shots > 0:
                blocks["fwi_large"] = run_fwi_large(a, device)
            if a.serve_requests > 0:
                blocks["serving"] = run_serving(a, device, peak)
        if jobs is not None:
            jobs.close()
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
        result.update(blocks)
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


def run_c0(a, device, peak, case, jobs):
    """The plain elastic forward of one shot: 600 x 300, DH 5 m, DT 0.4 ms, NT 5000,
    FDORDER 8, CPML 20, free surface, explosive Ricker 10 Hz at (1500 m, 10 m), 120
    receivers at z = 20 m.  Device time of the batched (graph-replayed) and of the
    plain (one launch per operation) path, the same end to end through the public
    API from host arrays, and the reference's own full run on one host core, whose
    sections the GPU's must equal bit for bit."""
    import denise_b200 as dn
    import torch
    from denise_b200 import synth

    p, model, src, rec = case if case is not None else synth.c0_case(seed=0)
    cells = p.nx * p.ny * p.nt
    m = dn.Model(p, *model, device=device)
    s = dn.Shot(m, *src, *rec)
    dn.run([s])
    torch.cuda.synchronize(device)
    ms = []
    for _ in range(3):
        dn.run([s])
        ms.append(dn.last_run_stats()[0])
    batched_ms = float(np.median(ms))
    secs = (s.sections(dn.SEC_VX), s.sections(dn.SEC_VY))
    pl = []
    for _ in range(2):
        dn.run_plain(s)
        pl.append(dn.last_run_stats()[0])
    plain_ms = float(np.median(pl))
    prof = dn.api.profile_steps([s], dn.MODE_FORWARD, nsteps=50)
    s.close()
    m.close()
    # end to end: host set-up and upload, the run, sections read back
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    m = dn.Model(p, *model, device=device)
    s = dn.Shot(m, *src, *rec)
    dn.run([s])
    out = (s.sections(dn.SEC_VX), s.sections(dn.SEC_VY))
    s.close()
    m.close()
    torch.cuda.synchronize(device)
    e2e_s = time.perf_counter() - t0
    h2d = 3 * model[0].nbytes + src[2].nbytes + 8 * len(rec[0])
    d2h = out[0].nbytes + out[1].nbytes
    blk = {"workload": f"plain elastic forward: one shot, {p.nx}x{p.ny} grid, DH {p.dh} m, DT {p.dt} s, NT {p.nt}, "
                       "FDORDER 8, FW 20, free surface, 120 receivers",
           "value": round(cells / (batched_ms * 1e-3) / 1e6, 1), "unit": UNIT,
           "ms_per_shot": round(batched_ms, 2),
           "plain_ms_per_shot": round(plain_ms, 2),
           "plain_value": round(cells / (plain_ms * 1e-3) / 1e6, 1),
           "shots_per_s": {"batched": round(1e3 / batched_ms, 3), "plain": round(1e3 / plain_ms, 3)},
           "whole_step_gbs_direct": round(80 * p.nx * p.ny / (sum(prof.values()) * 1e-3) / 1e9, 1),
           "e2e": {"value": round(cells / e2e_s / 1e6, 1), "unit": UNIT, "seconds": round(e2e_s, 3),
                   "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}}
    blk["whole_step_frac"] = round(blk["whole_step_gbs_direct"] / peak, 4)
    ref = jobs.result("c0") if jobs is not None else None
    if ref is not None:
        rvx, rvy, rsec = ref
        blk["cpu_baseline"] = {"value": round(cells / rsec / 1e6, 3), "unit": UNIT, "cores": 1, "kind": "reference",
                               "sample": "the reference's own full run of this shot (NT 5000) in one single-rank "
                                         f"process ({rsec:.1f} s, set-up included)"}
        blk["sections_bitwise_equal_reference"] = bool(np.array_equal(secs[0], rvx) and np.array_equal(secs[1], rvy))
    elif jobs is not None and "c0" in jobs.notes:
        blk["cpu_baseline"] = {"unavailable": jobs.notes["c0"]}
    return blk


def run_elastic(a, inputs, device, peak):
    """The same 64 shots (the 2000 x 600 grid of the batched workload) with the elastic
    propagator (vp, vs, rho of each model, L = 0) over the full NT = a.elastic_nt:
    device time of the batched run and the elastic step's per-kernel roofline."""
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
    ms = []
    with ClockSampler(device) as clk:
        for _ in range(2):
            dn.run(shots)
            ms.append(dn.last_run_stats()[0])
    ms = float(np.mean(ms))
    cells = len(shots) * p.nx * p.ny
    prof = dn.api.profile_steps(shots, dn.MODE_FORWARD, nsteps=20)
    step_ms = sum(prof.values())
    out = {"workload": f"batched elastic forward: {len(shots)} shots x {p.nx}x{p.ny} grid, NT={p.nt}, FDORDER 8, "
                       "FW 20, free surface, 400 receivers/shot (the models of the batched workload, L = 0)",
           "value": round(cells * p.nt / (ms * 1e-3) / 1e6, 1), "unit": UNIT, "shots": len(shots), "nt": p.nt,
           "ms_per_run": round(ms, 2),
           "v_kernel_gbs": round(36 * cells / (prof["update_v"] * 1e-3) / 1e9, 1),
           "s_kernel_gbs": round(44 * cells / (prof["update_s"] * 1e-3) / 1e9, 1),
           "whole_step_gbs_direct": round(80 * cells / (step_ms * 1e-3) / 1e9, 1),
           "kernel_ms": {k: round(v, 4) for k, v in prof.items()},
           "clocks": clk.summary()}
    out["whole_step_frac"] = round(out["whole_step_gbs_direct"] / peak, 4)
    out["v_kernel_frac"] = round(out["v_kernel_gbs"] / peak, 4)
    for m, s in pairs:
        s.close()
        m.close()
    return out


def run_gradient(a, device, c2in, jobs):
    """FWI gradient (forward with snapshots + adjoint) of the 1700 x 500 elastic workload:
    true model = the seeded family (seed 2), starting model = it smoothed with sigma 25
    cells, observed data synthesised on the GPU from the true model; FP16 snapshots
    every 2 steps; shots streamed through HBM in the batches shard.memory_batches
    gives (as many as 90 % of the free HBM holds, spread evenly).  On shot 0: the
    errors of the GPU's FP32 gradient against the reference's own and of its
    FP16-snapshot gradient against the FP64 restatement, both host runs timed."""
    import denise_b200 as dn
    import torch
    from denise_b200 import shard

    import config_cases as CC
    import oracles as O

    n = a.gradient_shots
    p, true, start, shots = CC.c2_case(nshots=n, snap_precision=dn.SNAP_F16)
    mt = dn.Model(p.replace(store_snapshots=0), *true, device=device)
    st_ = [dn.Shot(mt, *sh) for sh in shots]
    dn.run(st_)
    obs = [(s.sections(dn.SEC_VX), s.sections(dn.SEC_VY)) for s in st_]
    for s in st_:
        s.close()
    mt.close()

    def grad(params, idx):
        m = dn.Model(params, *start, device=device)
        L2, dev_ms, nb = 0.0, 0.0, []
        for part in shard.memory_batches(params, shots, idx, 1, device):
            nb.append(len(part))
            ss = [dn.Shot(m, *shots[k]) for k in part]
            dn.run(ss, dn.MODE_FORWARD)
            dev_ms += dn.last_run_stats()[0]
            for s, k in zip(ss, part):
                L2 += s.residual(obs[k][0], dn.SEC_VX) + s.residual(obs[k][1], dn.SEC_VY)
            dn.run(ss, dn.MODE_ADJOINT)
            dev_ms += dn.last_run_stats()[0]
            for s in ss:
                s.accumulate_gradient()
                s.close()
        g = m.gradient()
        m.close()
        return g, L2, dev_ms, nb

    grad(p, [0])                                   # warm-up (graphs, module load)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    g16, L2, dev_ms, nb = grad(p, list(range(n)))
    torch.cuda.synchronize(device)
    wall = time.perf_counter() - t0
    cells = n * p.nx * p.ny * p.nt * 2
    g32, _, _, _ = grad(p.replace(snap_precision=dn.SNAP_F32), [0, n // 2])
    g16s, _, _, _ = grad(p, [0, n // 2])
    err = max(O.rel_l2(x, y) for x, y in zip(g16s, g32))
    out = {"workload": f"FWI gradient, elastic {p.nx}x{p.ny}, DH {p.dh} m, DT {p.dt} s, NT {p.nt}, FDORDER 8, "
                       f"{n} shots x 400 receivers, FP16 snapshots every DTINV={p.dtinv} steps, "
                       "starting model smoothed sigma 25 cells, observed data synthesised on the GPU",
           "shots": n, "batches": nb, "seconds": round(wall, 2),
           "device_ms": round(dev_ms, 1), "shots_per_s": round(n / wall, 3),
           "mcell_updates_per_s": round(cells / wall / 1e6, 1),
           "misfit": L2, "fp16_vs_fp32_gradient_rel_l2": float(err)}
    if c2in is not None and jobs is not None:
        grads = c2in[5]
        cs = p.nx * p.ny * p.nt * 2
        ref = jobs.result("c2_ref")
        base = []
        if ref is not None:
            out["fp32_vs_reference_rel_l2"] = float(max(O.rel_l2(x, y) for x, y in zip(grads[dn.SNAP_F32], ref[:3])))
            out["fp32_bitwise_equal_reference"] = bool(all(np.array_equal(x, y)
                                                            for x, y in zip(grads[dn.SNAP_F32], ref[:3])))
            base.append({"value": round(cs / ref[4] / 1e6, 3), "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": "the reference's own gradient of shot 0 of this workload (forward with "
                                   f"snapshots, calc_res, adjoint, ass_gradPSV) in one process, {ref[4]:.0f} s"})
        f64 = jobs.result("c2_fp64")
        if f64 is not None:
            out["fp16_vs_fp64_oracle_rel_l2"] = float(max(O.rel_l2(x, y) for x, y in zip(grads[dn.SNAP_F16], f64[:3])))
            out["fp32_vs_fp64_oracle_rel_l2"] = float(max(O.rel_l2(x, y) for x, y in zip(grads[dn.SNAP_F32], f64[:3])))
            base.append({"value": round(cs / f64[3] / 1e6, 3), "unit": UNIT, "cores": 8, "kind": "port",
                         "sample": "the FP64 restatement of the scheme (oracle/psv_oracle) on shot 0, 8 threads, "
                                   f"{f64[3]:.0f} s"})
        if base:
            out["cpu_baseline"] = base
        for k in ("c2", "c2_ref", "c2_fp64"):
            if k in jobs.notes:
                out.setdefault("host_runs", {})[k] = jobs.notes[k]
    return out


def run_fwi_large(a, device):
    """A sample of the large FWI iteration: elastic 8000 x 2000, DH 2.5 m, DT 0.2 ms
    (0.25 ms breaks the CFL limit of this model), NT 12000, FDORDER 8, shots of the
    96-shot line with 1600 receivers; true model = the seeded family (seed 4) plus a
    5500 m/s ellipse, starting model smoothed with sigma 25 cells; one FWI iteration
    with FP16 snapshots every 4 steps and checkpointed adjoints (segments of 400
    steps) run as one batch, the reference's L-BFGS, the parabolic step search
    and the update."""
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
                        f"{n} of 96 shots x 1600 receivers in one batch, FP16 snapshots every 4 steps, checkpointed "
                        "adjoint (400-step segments), the reference's L-BFGS, parabolic step search",
            "shots": n, "setup_s": round(t1 - t0, 1), "observed_data_s": round(t2 - t1, 1),
            "forward_device_s_per_shot": round(per_shot_fwd, 2),
            "forward_mcell_updates_per_s": round(cells / per_shot_fwd / 1e6, 1),
            "gradient_s": round(h["gradient_s"], 1), "gradient_s_per_shot": round(per_shot_grad, 2),
            "gradient_mcell_updates_per_s": round(2 * cells * n / h["gradient_s"] / 1e6, 1),
            "optimizer_s": round(h["optimizer_s"], 3), "step_search_s": round(h["step_search_s"], 1),
            "test_models": h["test_models"], "step_found": h["found"], "eps": h["eps"],
            "misfit_before": L2, "misfit_after": L2_new,
            "iteration_s": round(t3 - t2, 1),
            "iteration_96_shots_estimate_s": round(96 * per_shot_grad + h["test_models"] * 96 * per_shot_fwd, 0)}


def _request_bytes(kind, p, nshots):
    """Algorithmic HBM bytes of a request: 80 B per elastic and (23 + 6L) 4 B per
    viscoelastic cell-update; a gradient adds its adjoint (96 B per cell-update)
    and per snapshot 5 s_b (store) plus 5 s_b + 8 + 6 g_b (correlation) bytes per
    cell, FP16 snapshots (s_b = 2) and float accumulators (g_b = 4)."""
    c = p.nx * p.ny
    fwd = (80 if p.L == 0 else (23 + 6 * p.L) * 4) * c * p.nt
    if kind != "gradient":
        return fwd * nshots
    nsnap = -(-p.nt // max(p.dtinv, 1))
    return (fwd + c * (96 * p.nt + nsnap * (10 + 10 + 8 + 24))) * nshots


def run_serving(a, device, peak):
    """The serving workload (2000 requests in the full stream; a.serve_requests of
    it here): requests of the mix arrive as a Poisson process at 1.2x the
    capacity of that mix, measured first by a closed-loop run of
    a.serve_calibration requests of another seed (all submitted at once); the
    server admits them by HBM footprint into its run queues.  Latency =
    scheduled arrival -> result on the host.  The HBM fraction is the mix's
    algorithmic bytes over the wall time of the stream."""
    from concurrent.futures import ThreadPoolExecutor

    from denise_b200 import serve, synth

    def make(n, seed):
        # the models of the stream are drawn in parallel threads (scipy releases the GIL)
        chunks = [(k, min(k + 16, n)) for k in range(0, n, 16)]
        with ThreadPoolExecutor(max_workers=8) as ex:
            parts = list(ex.map(lambda c: synth.serve_requests(n, seed=seed, scale=a.serve_scale, first=c[0],
                                                                 last=c[1]), chunks))
        return [r for part in parts for r in part]

    def drive(reqs, arrivals):
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
        return wall, st, bad

    cal = make(a.serve_calibration, 33)
    cal_wall, _, _ = drive(cal, np.zeros(len(cal)))
    capacity = len(cal) / cal_wall                                    # requests per second, closed loop
    cal_bytes = sum(_request_bytes(k, p, len(sh)) for k, p, _, sh, _ in cal)
    del cal
    reqs = make(a.serve_requests, 3)
    work = [p.nx * p.ny * p.nt * len(sh) * (2 if k == "gradient" else 1) for k, p, _, sh, _ in reqs]
    nbytes = sum(_request_bytes(k, p, len(sh)) for k, p, _, sh, _ in reqs)
    rate = 1.2 * capacity
    rng = np.random.default_rng(3)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
    wall, st, bad = drive(reqs, arrivals)
    return {"requests": len(reqs), "failed": bad, "p50_latency_s": round(st["p50_s"], 3),
            "p99_latency_s": round(st["p99_s"], 3), "shots_per_s": round(st["shots_done_total"] / wall, 3),
            "mcell_updates_per_s": round(sum(work) / wall / 1e6, 1), "wall_s": round(wall, 2),
            "hbm_gbs": round(nbytes / wall / 1e9, 1), "hbm_frac": round(nbytes / wall / 1e9 / peak, 4),
            "arrival_rate_per_s": round(rate, 3),
            "capacity": {"requests_per_s": round(capacity, 3), "requests": a.serve_calibration,
                         "wall_s": round(cal_wall, 2), "hbm_frac": round(cal_bytes / cal_wall / 1e9 / peak, 4),
                         "how": "closed loop: all requests of a seed-33 stream submitted at once"},
            "max_running_shots": st["max_running_shots"], "joins_while_running": st["joins_while_running"],
            "workload": "seeded serving mix: 70% elastic forward, 20% visco L=3 forward, 10% elastic FWI gradient "
                        "(FP16 snapshots); NX 300-3000, NZ 150-1000, NT 2000-8000 (x scale "
                        f"{a.serve_scale}), FDORDER 4/8/12, 1-4 shots, 50-500 receivers; Poisson arrivals at 1.2x "
                        "the measured capacity of the mix; the first "
                        f"{a.serve_requests} of the 2000-request stream"}


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
            "config": dict(workload_config(a, p, world, ours=False), parallelism="host processes",
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
