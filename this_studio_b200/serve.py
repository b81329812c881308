"""Served form: a request loop that admits independent scenes while others
run, by HBM budget, into the batched form (this_studio_b200/batch.py).

Requests arrive over time (a seeded Poisson stream of DEM drops and WCSPH
dam breaks of uneven size).  The server keeps one DEM batch and one WCSPH
batch resident on the GPU, each on its own CUDA stream and host thread so the
two overlap on the device.  Every chunk of steps (a multiple of 5 for DEM, the
re-sort cadence) it retires finished members, admits waiting requests whose
memory estimate fits the budget, and rebuilds the batch with the continuing
members' state carried over.  Reported: aggregate particle-steps/s, p50 / p99
of scene latency (arrival to completion) and of scene-step latency (wall time
of the chunk a scene-step ran in, divided by the chunk's steps), and admission
waits.
"""
from __future__ import annotations

import math
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import scenes
from .batch import DEMBatch, Member, SPHBatch

# device bytes per particle (state + lists at their usual capacities)
DEM_BYTES_PER_BALL = 2400
SPH_BYTES_PER_FLUID = 900
SPH_BYTES_PER_DUMMY = 200


@dataclass
class Request:
    key: int
    kind: str          # "dem" or "sph"
    n: int             # requested particle count
    steps: int
    arrival: float     # seconds after the stream starts
    seed: int
    scene: object = None
    admitted: float = None
    done: float = None
    np_: int = 0       # particles actually generated
    final: dict = None # member state at completion (kept when the server keeps states)
    step_lat: list = field(default_factory=list)

    def build(self, sph_c0, sph_dt):
        if self.scene is None:
            if self.kind == "dem":
                self.scene = scenes.dem_drop_poly(self.n, self.seed)
            else:
                self.scene = scenes.sph_column(self.n, sph_c0, sph_dt)
        return self.scene

    def particles(self):
        sc = self.scene
        return sc.position.shape[0] if self.kind == "dem" else sc.fluid.shape[0]

    def bytes(self):
        sc = self.scene
        if self.kind == "dem":
            return sc.position.shape[0] * DEM_BYTES_PER_BALL
        return sc.fluid.shape[0] * SPH_BYTES_PER_FLUID + sc.dummy.shape[0] * SPH_BYTES_PER_DUMMY


def stream_params(n_max, dx=0.01):
    """Sound speed and time step shared by all dam breaks of a stream: those
    of its tallest column, c0 = 10 sqrt(2 g H), dt = 0.25 h / (c0 + 2 sqrt(g H))."""
    g = 9.81
    nx = max(2, int(round((n_max / 2.0) ** (1.0 / 3.0))))
    H = 2 * nx * dx
    c0 = 10.0 * math.sqrt(2 * g * H)
    return c0, 0.25 * 1.3 * dx / (c0 + 2.0 * math.sqrt(g * H))


def make_stream(num, seed=7, n_min=1000, n_max=200_000, rate=50.0, steps=500, kinds=("dem", "sph")):
    """num requests, Poisson arrivals at `rate` per second, kind uniform over
    `kinds`, particle count log-uniform over [n_min, n_max]."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=num))
    out = []
    for k in range(num):
        n = int(math.exp(rng.uniform(math.log(n_min), math.log(n_max))))
        out.append(Request(key=k, kind=str(rng.choice(kinds)), n=n, steps=steps, arrival=float(t[k]),
                           seed=int(rng.integers(1 << 30))))
    return out


def _pct(v, q):
    return float(np.percentile(np.asarray(v, float), q)) if len(v) else None


class SceneServer:
    def __init__(self, hbm_budget=40e9, chunk=50, precision="mixed", max_members=512, sph_c0=None, sph_dt=None,
                 keep_states=False):
        import torch

        assert chunk % 5 == 0, "chunks are a multiple of the DEM re-sort cadence"
        self.torch = torch
        self.budget = hbm_budget
        self.chunk = chunk
        self.precision = precision
        self.max_members = max_members
        self.keep_states = keep_states
        self.sph_c0, self.sph_dt = sph_c0, sph_dt
        self.streams = {"dem": torch.cuda.Stream(), "sph": torch.cuda.Stream()}
        self.batches = {"dem": DEMBatch(precision, self.streams["dem"]),
                        "sph": SPHBatch(precision, self.streams["sph"])}

    def run(self, requests, log=None):
        reqs = sorted(requests, key=lambda r: r.arrival)
        if self.sph_c0 is None:
            self.sph_c0, self.sph_dt = stream_params(max(r.n for r in reqs))
        waiting = list(reqs)
        active = {"dem": {}, "sph": {}}
        used = 0.0
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        busy = 0.0
        chunks = 0
        rebuild_s = 0.0
        retired = {"dem": {}, "sph": {}}
        while waiting or active["dem"] or active["sph"]:
            t = now()
            # retire
            for kind in ("dem", "sph"):
                b = self.batches[kind]
                for m in b.members:
                    if m.key in active[kind] and m.steps_done >= active[kind][m.key].steps:
                        r = active[kind].pop(m.key)
                        r.done = t
                        used -= r.bytes()
                        r.scene = None
                        retired[kind][m.key] = r
            # admit (arrival order, first fit by budget)
            changed = {"dem": False, "sph": False}
            keep = []
            for r in waiting:
                if r.arrival <= t and len(active[r.kind]) < self.max_members:
                    r.build(self.sph_c0, self.sph_dt)
                    r.np_ = r.particles()
                    if used + r.bytes() <= self.budget or not (active["dem"] or active["sph"]):
                        used += r.bytes()
                        r.admitted = t
                        active[r.kind][r.key] = r
                        changed[r.kind] = True
                        continue
                keep.append(r)
            waiting = keep
            # rebuild batches whose membership changed, carrying state
            tr = time.perf_counter()
            for kind in ("dem", "sph"):
                b = self.batches[kind]
                cur = {m.key for m in b.members}
                want = set(active[kind])
                if cur != want or changed[kind]:
                    b.capture()
                    old = {m.key: m for m in b.members}
                    for k in cur - want:
                        if self.keep_states:
                            retired[kind][k].final = old[k].state
                        retired[kind].pop(k, None)
                    b.members = [old[k] if k in old else Member(key=k, scene=active[kind][k].scene)
                                 for k in sorted(want)]
                    b.rebuild()
            rebuild_s += time.perf_counter() - tr
            if not (active["dem"] or active["sph"]):
                if waiting:  # idle until the next arrival
                    time.sleep(max(0.0, min(0.05, waiting[0].arrival - now())))
                continue
            # one chunk on both batches at once (separate streams and threads)
            c0 = time.perf_counter()
            lat = {}

            def run(kind):
                b = self.batches[kind]
                if b.members:
                    s = time.perf_counter()
                    b.step(self.chunk)
                    lat[kind] = (time.perf_counter() - s) / self.chunk

            th = [threading.Thread(target=run, args=(k,)) for k in ("dem", "sph")]
            for x in th:
                x.start()
            for x in th:
                x.join()
            busy += time.perf_counter() - c0
            chunks += 1
            for kind, l in lat.items():
                for r in active[kind].values():
                    r.step_lat.append(l)
            if log:
                log(f"t={now():.2f}s active dem={len(active['dem'])} sph={len(active['sph'])} "
                    f"waiting={len(waiting)} lat={lat}")
        makespan = now()
        for b in self.batches.values():
            b.solver = None
        return self._metrics(reqs, makespan, busy, chunks, rebuild_s)

    def _metrics(self, reqs, makespan, busy, chunks, rebuild_s):
        ps = sum(r.np_ * r.steps for r in reqs)
        lat = [r.done - r.arrival for r in reqs]
        wait = [r.admitted - r.arrival for r in reqs]
        steplat = [x for r in reqs for x in r.step_lat]
        return {"scenes": len(reqs), "particle_steps": ps, "value": ps / makespan, "value_busy": ps / busy,
                "makespan_s": makespan, "busy_s": busy, "chunks": chunks,
                "rebuild_s": rebuild_s,
                "scene_latency_p50_s": _pct(lat, 50), "scene_latency_p99_s": _pct(lat, 99),
                "scene_step_latency_p50_ms": 1e3 * _pct(steplat, 50), "scene_step_latency_p99_ms": 1e3 * _pct(steplat, 99),
                "admission_wait_p50_s": _pct(wait, 50), "admission_wait_p99_s": _pct(wait, 99)}


def particle_steps(requests, sph_c0, sph_dt):
    """Total particle-steps of a stream (moving DEM spheres + SPH fluid)."""
    tot = 0
    for r in requests:
        had = r.scene is not None
        sc = r.build(sph_c0, sph_dt)
        tot += (sc.position.shape[0] if r.kind == "dem" else sc.fluid.shape[0]) * r.steps
        if not had:
            r.scene = None
    return tot


def run_plain(requests, precision="mixed", sph_c0=None, sph_dt=None):
    """Every request alone on the plain solver, one after another."""
    import torch

    if sph_c0 is None:
        sph_c0, sph_dt = stream_params(max(r.n for r in requests))
    t0 = time.perf_counter()
    for r in requests:
        sc = r.build(sph_c0, sph_dt)
        s = scenes.build_dem(sc, precision) if r.kind == "dem" else scenes.build_sph(sc, precision)
        s.step(r.steps)
        del s
        r.scene = None
    torch.cuda.synchronize()
    return time.perf_counter() - t0
