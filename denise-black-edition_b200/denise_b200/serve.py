"""Request serving with continuous batching on one GPU.

Requests (forward modelling or FWI gradient, any grid size) are admitted by
their HBM footprint (dn_model_footprint + dn_shot_footprint of every shot);
admitted requests keep models and wavefields device-resident until their
result is on the host.  Shots run in run queues (dn_queue_*), one per FDORDER,
L and arithmetic: a queue advances all its shots together in chunks of time
steps, each shot at its own time step, and admits new shots between chunks, so
requests that arrive while others are on the GPU join the running batch.
Queues own CUDA streams, so the work of different classes overlaps.

A gradient request runs each shot forward with snapshot storage, forms the L2
residual against the request's observed data on the device (calc_res, LNORM
2), runs the adjoint in the same queue and stacks the shot's gradient into the
model's gradient (ass_gradPSV).  Latency is arrival to result on the host.
"""
import ctypes
import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, lib
from .api import Model, Shot, PsvParams


@dataclass
class Request:
    """One request.  shots: list of (src_i, src_j, signals, rec_i, rec_j[, src_type, src_azi]);
    obs (gradient only): per shot (obs_vx, obs_vy), each [ntr][nt]."""

    kind: str                      # "forward" or "gradient"
    params: PsvParams
    model: tuple                   # (vp, vs, rho[, qp, qs]) as (nx, ny) float32, file order
    shots: list
    obs: list = None
    rid: int = 0
    arrival: float = 0.0


@dataclass
class Result:
    rid: int
    kind: str
    status: int
    latency_s: float
    sections: list = None          # forward: per shot {"vx": [ntr][nt], "vy": ...}
    gradient: tuple = None         # gradient: (g_vp, g_vs, g_rho) in file order
    misfit: float = 0.0


def footprint(req):
    """HBM bytes a request holds while it runs: its model plus all its shots."""
    p = req.params.to_c()
    b = ctypes.c_size_t()
    check(lib.dn_model_footprint(ctypes.byref(p), ctypes.byref(b)))
    total = b.value
    store = 1 if req.kind == "gradient" else 0
    for sh in req.shots:
        check(lib.dn_shot_footprint(ctypes.byref(p), len(sh[3]), store, ctypes.byref(b)))
        total += b.value
    return total


def plan_admission(waiting, free_bytes, head_wait, max_head_wait):
    """Which waiting requests to admit now, in arrival order.

    waiting: footprints in arrival order.  First fit: every request that fits in
    what is left is admitted; but once the head of the line has waited
    max_head_wait rounds, nothing behind it is admitted until it fits, so a
    large request cannot be starved by a stream of small ones."""
    take, left = [], free_bytes
    for k, fp in enumerate(waiting):
        if fp <= left:
            take.append(k)
            left -= fp
        elif k == 0 and head_wait >= max_head_wait:
            break
    return take


class _Live:
    """An admitted request and its device objects."""

    def __init__(self, req, fp, device):
        self.req, self.fp = req, fp
        p = req.params
        mdl = req.model
        self.model = Model(p, *mdl[:3], mdl[3] if p.L else None, mdl[4] if p.L else None, device=device)
        store = req.kind == "gradient"
        self.shots = []
        for sh in req.shots:
            kw = {}
            if len(sh) > 5:
                kw = dict(src_type=sh[5], src_azi=sh[6])
            self.shots.append(Shot(self.model, sh[0], sh[1], sh[2], sh[3], sh[4], **kw))
        self.left = len(self.shots)
        self.sections = [None] * len(self.shots)
        self.misfits = [0.0] * len(self.shots)
        self.status = 0
        self.store = store

    def close(self):
        for s in self.shots:
            s.close()
        self.model.close()


class Server:
    def __init__(self, device=0, hbm_budget=None, chunk=50, max_head_wait=8):
        self.device = device
        self.chunk = chunk
        self.max_head_wait = max_head_wait
        if hbm_budget is None:
            free, total = ctypes.c_size_t(), ctypes.c_size_t()
            check(lib.dn_device_memory(device, ctypes.byref(free), ctypes.byref(total)))
            hbm_budget = int(0.85 * free.value)
        self.budget = hbm_budget
        self.used = 0
        self.waiting = []              # (req, footprint)
        self.head_wait = 0
        self.queues = {}               # class key -> dn_queue handle
        self.owner = {}                # shot handle value -> (live, shot index)
        self.results = []
        self.rounds = 0
        self.max_running = 0
        self.joins_while_running = 0
        self.shots_done = 0
        self._t0 = None

    # -- submission -----------------------------------------------------------------------------
    def submit(self, req, now=None):
        req.arrival = time.perf_counter() if now is None else now
        if self._t0 is None:
            self._t0 = req.arrival
        fp = footprint(req)
        if fp > self.budget:
            raise _lib.DeniseError(_lib.DN_ENOMEM, f"request {req.rid} needs {fp} B, more than the budget")
        self.waiting.append((req, fp))

    def idle(self):
        return not self.waiting and not self.owner

    # -- one scheduling round ---------------------------------------------------------------------
    def step(self):
        self.rounds += 1
        self._admit()
        for key, q in list(self.queues.items()):
            self._step_queue(q)
        return self.idle()

    def run(self):
        while not self.idle():
            self.step()
        return self.results

    def _queue(self, p):
        key = (p.fdorder, p.L, p.arith)
        if key not in self.queues:
            h = _lib._vp()
            check(lib.dn_queue_create(self.device, self.chunk, ctypes.byref(h)))
            self.queues[key] = h
        return self.queues[key]

    def _admit(self):
        if not self.waiting:
            return
        take = plan_admission([fp for _, fp in self.waiting], self.budget - self.used, self.head_wait,
                              self.max_head_wait)
        if take and take[0] == 0:
            self.head_wait = 0
        elif self.waiting:
            self.head_wait += 1
        chosen = set(take)
        admitted = [self.waiting[k] for k in take]
        self.waiting = [w for k, w in enumerate(self.waiting) if k not in chosen]
        for req, fp in admitted:
            live = _Live(req, fp, self.device)
            self.used += fp
            q = self._queue(req.params)
            running = ctypes.c_int()
            check(lib.dn_queue_count(q, ctypes.byref(running), None))
            if running.value > 0:
                self.joins_while_running += 1
            for i, s in enumerate(live.shots):
                self.owner[s.handle.value] = (live, i)
                check(lib.dn_queue_add(q, s.handle, _lib.MODE_FORWARD))

    def _step_queue(self, q):
        cap = 256
        done = (_lib._vp * cap)()
        status = (ctypes.c_int * cap)()
        nd = ctypes.c_int()
        while True:
            check(lib.dn_queue_step(q, done, status, cap, ctypes.byref(nd)))
            for k in range(nd.value):
                self._finished(q, done[k], status[k])
            running = ctypes.c_int()
            check(lib.dn_queue_count(q, ctypes.byref(running), None))
            self.max_running = max(self.max_running, running.value)
            if nd.value < cap:
                break

    def _finished(self, q, h, st):
        live, i = self.owner[h]
        shot = live.shots[i]
        mode = getattr(shot, "_serve_mode", 0)
        if st != 0:
            live.status = st
        if live.req.kind == "forward" or st != 0:
            if st == 0:
                live.sections[i] = {"vx": shot.sections(_lib.SEC_VX), "vy": shot.sections(_lib.SEC_VY)}
            self._shot_done(live, h)
            return
        if mode == 0:
            ovx, ovy = live.req.obs[i]
            live.misfits[i] = shot.residual(ovx, _lib.SEC_VX) + shot.residual(ovy, _lib.SEC_VY)
            shot._serve_mode = 1
            check(lib.dn_queue_add(q, h, _lib.MODE_ADJOINT))
            return
        self._shot_done(live, h)

    def _shot_done(self, live, h):
        del self.owner[h]
        self.shots_done += 1
        live.left -= 1
        if live.left:
            return
        res = Result(live.req.rid, live.req.kind, live.status, 0.0)
        if live.status == 0:
            if live.req.kind == "forward":
                res.sections = live.sections
            else:
                # stacked in shot order whatever order the shots finished in, so the
                # float sums are those of a run of the request alone
                for shot in live.shots:
                    shot.accumulate_gradient()
                res.gradient = live.model.gradient()
                res.misfit = float(sum(live.misfits))
        res.latency_s = time.perf_counter() - live.req.arrival
        self.results.append(res)
        self.used -= live.fp
        live.close()

    # -- statistics -----------------------------------------------------------------------------
    def stats(self):
        lat = np.array([r.latency_s for r in self.results]) if self.results else np.zeros(1)
        wall = time.perf_counter() - (self._t0 or time.perf_counter())
        return {"requests": len(self.results), "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "shots_per_s": self.shots_done / max(wall, 1e-9),
                "max_running_shots": self.max_running, "joins_while_running": self.joins_while_running,
                "rounds": self.rounds, "shots_done_total": self.shots_done}

    def close(self):
        for q in self.queues.values():
            lib.dn_queue_destroy(q)
        self.queues = {}
