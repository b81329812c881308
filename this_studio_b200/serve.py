"""Served form: a request loop that admits independent scenes while others
run, by HBM budget, into the batched form (this_studio_b200/batch.py).

Requests arrive over time (a seeded Poisson stream of DEM drops and WCSPH
dam breaks of uneven size); each carries its scene, generated before the
clock starts, as a client would send it.  The server keeps one DEM batch and
one WCSPH batch resident on the GPU, each on its own CUDA stream and host
thread so the two overlap on the device.  Every chunk of steps (a multiple of
5 for DEM, the re-sort cadence) a kind's worker retires finished members,
admits waiting requests whose memory estimate fits the budget, and rebuilds
its batch with the continuing members' state carried over on the device.  Reported: aggregate particle-steps/s, p50 / p99
of scene latency (arrival to completion) and of scene-step latency (wall time
of the chunk a scene-step ran in, divided by the chunk's steps), admission
waits, and per kind the seconds its batch was stepping, waiting for the next
batch scene to be prepared, and idle with nothing admitted.
"""
from __future__ import annotations

import math
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import scenes
from .batch import DEMBatch, Member, SPHBatch

# device bytes per particle: state, lists at their usual capacities and the
# step's snapshot for overflow replay (measured on a B200: 5.2 kB per ball of a
# 195k-ball drop, 2.6 kB per fluid particle of a 195k-particle dam break with
# as many dummies), with some headroom
DEM_BYTES_PER_BALL = 5600
SPH_BYTES_PER_FLUID = 1800
SPH_BYTES_PER_DUMMY = 900


@dataclass
class Request:
    key: int
    kind: str          # "dem" (drop), "dem_bonded" (agglomerates and clumps) or "sph"
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
            elif self.kind == "dem_bonded":
                self.scene = scenes.dem_agglomerate_drop(self.n, self.seed)
            else:
                self.scene = scenes.sph_column(self.n, sph_c0, sph_dt)
        return self.scene

    @property
    def batch_kind(self):
        """The batch that runs it: DEM kinds share one (same time step and gravity)."""
        return "sph" if self.kind == "sph" else "dem"

    def particles(self):
        """Moving particles: DEM balls and pebbles, SPH fluid."""
        sc = self.scene
        return sc.num_moving if self.batch_kind == "dem" else sc.fluid.shape[0]

    def bytes(self):
        sc = self.scene
        if self.batch_kind == "dem":
            return (sc.position.shape[0] + sum(len(c["radius"]) for c in sc.clumps)) * DEM_BYTES_PER_BALL
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
                 keep_states=False, autotune=False, tunings=None, batches=None):
        """batches: kind -> an object with the batch interface (members,
        timing, prepare, commit, step, capture, clear) in place of the device
        batches; the scheduling then runs without a GPU."""
        assert chunk % 5 == 0, "chunks are a multiple of the DEM re-sort cadence"
        self.budget = hbm_budget
        self.chunk = chunk
        self.precision = precision
        self.max_members = max_members
        self.keep_states = keep_states
        # autotune: tune each kind before serving (autotune.py) unless
        # `tunings` (kind -> autotune.Tuning, e.g. an earlier server's) is given
        self.autotune = autotune
        self.tunings = dict(tunings or {})
        self.sph_c0, self.sph_dt = sph_c0, sph_dt
        if batches is not None:
            self.streams = {}
            self.batches = dict(batches)
            return
        import torch

        from . import _lib

        # batches are re-created at membership changes: keep their memory pooled
        _lib.retain_device_memory(int(2 * hbm_budget))
        # two streams per kind: the next batch scene is prepared on one while
        # the current scene steps on the other.  The DEM step is many short
        # kernels and the SPH step a few long ones; the DEM streams get the
        # higher priority so their blocks are scheduled as SMs free up instead
        # of queueing behind whole SPH kernels.
        lo, hi = torch.cuda.Stream.priority_range() if hasattr(torch.cuda.Stream, "priority_range") else (0, -1)
        self.streams = {"dem": [torch.cuda.Stream(priority=hi), torch.cuda.Stream(priority=hi)],
                        "sph": [torch.cuda.Stream(priority=lo), torch.cuda.Stream(priority=lo)]}
        self.batches = {"dem": DEMBatch(precision, streams=self.streams["dem"], tuning=self.tunings.get("dem")),
                        "sph": SPHBatch(precision, streams=self.streams["sph"], tuning=self.tunings.get("sph"))}

    def run(self, requests, log=None):
        """Serves the requests to completion; returns the stream's metrics.

        One worker thread per kind owns that kind's batch.  Before each chunk
        a worker retires the members that finished, commits the batch scene
        prepared during the previous chunk (carrying the continuing members'
        state on the device), and plans the membership after the coming
        chunk: the members that will still be running plus arrived requests
        of its kind (arrival order, first fit against the shared HBM budget).
        If that differs from the current membership, the next batch scene is
        built and initialised on a helper thread and the batch's other stream
        while the chunk runs, so scene set-up overlaps the steps.  The
        prepared and the running scene coexist, so the device holds up to
        twice the budget at a boundary."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        if self.sph_c0 is None:
            self.sph_c0, self.sph_dt = stream_params(max(r.n for r in reqs))
        for r in reqs:
            r.build(self.sph_c0, self.sph_dt)
            r.np_ = r.particles()
        by_key = {r.key: r for r in reqs}
        tune_s = self._tune(reqs) if self.autotune and not self.tunings else 0.0
        lock = threading.Lock()
        waiting = {k: [r for r in reqs if r.batch_kind == k] for k in ("dem", "sph")}
        active = {"dem": {}, "sph": {}}
        used = [0.0]
        stats = {k: {"busy": 0.0, "chunks": 0, "rebuild": 0.0, "wait": 0.0, "idle": 0.0} for k in ("dem", "sph")}
        errors = []
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0

        def worker(kind):
            b = self.batches[kind]
            st = stats[kind]
            act = active[kind]
            prep = None      # (Prepared or None for "no members", newly admitted requests)
            try:
                while True:
                    # retire members that completed their steps
                    t = now()
                    gone = [m.key for m in b.members if m.steps_done >= by_key[m.key].steps]
                    if gone:
                        if self.keep_states:
                            b.capture(keys=set(gone))
                        with lock:
                            for k in gone:
                                r = by_key[k]
                                r.done = t
                                used[0] -= r.bytes()
                                del act[k]
                        for m in b.members:
                            if m.key in gone:
                                by_key[m.key].final = m.state if self.keep_states else None
                                by_key[m.key].scene = None
                    # commit the scene prepared during the last chunk
                    if prep is not None:
                        tr = time.perf_counter()
                        pr, adm = prep
                        prep = None
                        if pr is None:
                            b.clear()
                        else:
                            b.commit(pr)
                        st["rebuild"] += time.perf_counter() - tr
                        for r in adm:
                            r.admitted = now()
                    # plan the membership after the coming chunk
                    with lock:
                        surv = [m for m in b.members if m.steps_done + self.chunk < by_key[m.key].steps]
                        adm, keep = [], []
                        for r in waiting[kind]:
                            if r.arrival <= t and len(surv) + len(adm) < self.max_members and (
                                    used[0] + r.bytes() <= self.budget or not (active["dem"] or active["sph"])):
                                used[0] += r.bytes()
                                act[r.key] = r
                                adm.append(r)
                            else:
                                keep.append(r)
                        waiting[kind] = keep
                        pending = list(keep)
                    nxt = surv + [Member(key=r.key, scene=r.scene) for r in adm]
                    if not b.members:
                        if nxt:  # nothing running: set up now
                            tr = time.perf_counter()
                            b.commit(b.prepare(nxt))
                            st["rebuild"] += time.perf_counter() - tr
                            for r in adm:
                                r.admitted = now()
                            continue
                        if not pending:
                            return
                        ti = time.perf_counter()
                        time.sleep(max(0.0, min(0.02, pending[0].arrival - now())))
                        st["idle"] += time.perf_counter() - ti
                        continue
                    helper = None
                    out = []
                    if adm or len(surv) != len(b.members):
                        if nxt:
                            def build(ms=nxt):
                                try:
                                    out.append(b.prepare(ms))
                                except BaseException as e:
                                    out.append(e)

                            helper = threading.Thread(target=build)
                            helper.start()
                        else:
                            prep = (None, [])
                    c = time.perf_counter()
                    b.step(self.chunk)
                    lat = (time.perf_counter() - c) / self.chunk
                    st["busy"] += time.perf_counter() - c
                    st["chunks"] += 1
                    for m in b.members:
                        by_key[m.key].step_lat.append(lat)
                    if helper is not None:
                        tw = time.perf_counter()
                        helper.join()
                        st["wait"] += time.perf_counter() - tw
                        if isinstance(out[0], BaseException):
                            raise out[0]
                        prep = (out[0], adm)
                    if log:
                        log(f"t={now():.2f}s {kind}: members={len(b.members)} next={len(nxt)} "
                            f"waiting={len(pending)} lat={lat * 1e3:.3f} ms")
            except BaseException as e:  # surfaced on the calling thread
                errors.append(e)

        th = [threading.Thread(target=worker, args=(k,)) for k in ("dem", "sph")]
        for x in th:
            x.start()
        for x in th:
            x.join()
        if errors:
            raise errors[0]
        makespan = now()
        for b in self.batches.values():
            b.clear()
        busy = max(stats[k]["busy"] for k in stats)
        m = self._metrics(reqs, makespan, busy, sum(stats[k]["chunks"] for k in stats),
                          sum(stats[k]["rebuild"] for k in stats))
        kind_ps = {k: sum(r.np_ * r.steps for r in reqs if r.batch_kind == k) for k in stats}
        m["per_kind"] = {k: {"busy_s": stats[k]["busy"], "chunks": stats[k]["chunks"],
                             "commit_s": stats[k]["rebuild"], "particle_steps": kind_ps[k],
                             "prepare_wait_s": stats[k]["wait"], "idle_s": stats[k]["idle"],
                             **self.batches[k].timing} for k in stats}
        if self.tunings:
            m["tuning"] = {k: t.as_dict() for k, t in self.tunings.items()}
            m["tune_s"] = tune_s  # 0 when the tunings were given
        return m

    def _tune(self, reqs):
        """Autotunes each kind once, before serving, on the scene at the
        particle-weighted median of its first requests (the size that
        carries the kind's work; autotune.tune_dem / tune_sph); the batches
        then build every scene with the tuning.  Returns the seconds spent."""
        from . import autotune

        tic = time.perf_counter()
        for kind in ("dem", "sph"):
            early = [r for r in reqs[:64] if r.kind == kind] or [r for r in reqs if r.batch_kind == kind]
            if not early:
                continue
            early = sorted(early, key=lambda x: x.n)
            w = np.cumsum([x.n for x in early])
            r = early[int(np.searchsorted(w, 0.5 * w[-1]))]
            t = (autotune.tune_dem(r.scene, self.precision) if kind == "dem"
                 else autotune.tune_sph(r.scene, self.precision))
            self.tunings[kind] = t
            self.batches[kind].tuning = t
        return time.perf_counter() - tic

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
        tot += (sc.num_moving if r.batch_kind == "dem" else sc.fluid.shape[0]) * r.steps
        if not had:
            r.scene = None
    return tot


def run_plain(requests, precision="mixed", sph_c0=None, sph_dt=None, per_kind=None):
    """Every request alone on the plain solver, one after another.  Scenes
    are generated before the clock starts, as for the server; the time covers
    building each device scene (upload, initialisation) and its steps.  With
    a dict `per_kind`, each kind's seconds and particle-steps are added to it
    (per_kind[kind] = [seconds, particle-steps])."""
    import torch

    if sph_c0 is None:
        sph_c0, sph_dt = stream_params(max(r.n for r in requests))
    for r in requests:
        r.build(sph_c0, sph_dt)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in requests:
        sc = r.scene
        tk = time.perf_counter()
        s = scenes.build_dem(sc, precision) if r.batch_kind == "dem" else scenes.build_sph(sc, precision)
        s.step(r.steps)
        if per_kind is not None:
            torch.cuda.synchronize()
            e = per_kind.setdefault(r.batch_kind, [0.0, 0])
            e[0] += time.perf_counter() - tk
            e[1] += (sc.num_moving if r.batch_kind == "dem" else sc.fluid.shape[0]) * r.steps
        del s
        r.scene = None
    torch.cuda.synchronize()
    return time.perf_counter() - t0
