"""Benchmark of the DEMSPH particle-interaction path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Workload: the plain 3-D WCSPH dam break -- 128,000 fluid particles
(40 x 40 x 80 at dx = 0.01 m in a 0.4 x 0.4 x 0.8 m column) in a 1.6 x 0.4 x
1.0 m tank with 3 layers of dummy wall particles (150,216), Wendland C2 with
h = 1.3 dx, c0 = 10 sqrt(2 g 0.8), dt = 0.25 h / (c0 + 2 sqrt(0.8 g)).  One
step = the reference's WCSPH step: cell sort + neighbour lists, momentum,
kick, drift, continuity + EOS, momentum, kick.  Metric: particle-steps/s
(fluid particles x steps / second).

* value: K steps through the native C ABI with the state resident in HBM,
  each step bracketed by CUDA events on the launching stream; L2 (126 MB) is
  flushed by writing a 256 MB buffer between timed steps, outside the events.
* e2e: the same metric through the public solver API as a user runs it:
  scene upload from host memory, K steps, final state read back, all timed.
* roofline: the momentum kernel (the dominant one), timed live per launch,
  against the compulsory bytes of one pass of the mixed-precision design,
  with the FP32-SIMT and instruction-issue fractions beside it.
* dem: the plain 4,096-sphere bounce, its contact-rich form and the bonded
  beam + clumps, each with its roofline (measured pair and bond counts).
* reference_cuda: the reference's own CUDA kernels on the same workloads.
* conservation_fp64: device FP64 diagnostics of the fluid around the timed steps.
* stream: the serving / batching stream -- 2,000 seeded scenes (DEM drops
  and WCSPH dam breaks, 1k-200k particles, 500 steps each, Poisson arrivals)
  through the continuous-batching server in mixed precision, beside the same
  scenes run one at a time on the plain solver (mixed; FP64 on a prefix);
  wall clock, with p50 / p99 scene-step and scene latency, admission waits.
* cpu_baseline: the FP64 C++ oracle on the host cores over a short sample.
* --impl reference: the reference's step restated as the FP64 C++ oracle
  (the reference has no CPU path; its CUDA build cannot be installed as a
  package) on all host cores, same workload and metric.

Multi-GPU: replicas only (one independent scene per rank, no collective on
the data path); value = all ranks' particle-steps / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s"
WORKLOAD = "wcsph_dam_break_128k"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--stress", type=int, default=1,
                    help="1: also time the bonded beam + clumps and the coupled ice sheet (about 40 s more)")
    ap.add_argument("--stream", type=int, default=2000,
                    help="scenes in the served-stream measurement (0: skip it)")
    return ap.parse_args()


# ---------------------------------------------------------------- clocks --
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        mhz = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k] == "Active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ------------------------------------------------------------ workload ----
def workload():
    from this_studio_b200 import scenes

    return scenes.sph_dam_break()


def sph_bytes_8d(nf, nd, ncell):
    """Compulsory HBM bytes of one WCSPH step of the mixed-precision design
    (the per-step model of the hot-path measurement plan): three passes each
    reading x, v (FP64) and rho, p, c, h, m, nu (FP32) per particle (72 B);
    their outputs a, a, drho-rate (12 + 12 + 4 B); the integration's
    read-modify-write of v, x, drho (48 + 48 + 16 B); the per-step re-key and
    sort (24 + 8 + 16 B); the dummies read twice (24 B); the cell table (8 B
    per cell).  Lists and neighbour re-reads are not counted."""
    return 3 * nf * 72 + nf * (12 + 12 + 4) + nf * (48 + 48 + 16) + nf * (24 + 8 + 16) + nd * 24 * 2 + ncell * 8


def momentum_bytes_8d(nf, nd):
    """The same model for one momentum pass: each fluid particle's 72 B read
    and its 12 B acceleration written, each dummy's 24 B read."""
    return nf * (72 + 12) + nd * 24


def dem_bytes_8d(n, pairs, springs, bonds):
    """Compulsory HBM bytes of one DEM step of the mixed-precision design:
    two force passes reading 88 B and writing 24 B per particle, 288 B of
    integration per particle, per contact pair 8 B of ids and 48 B per active
    spring kind read-modify-written in each pass, 192 B per bond per pass,
    and every fifth step the rebuild (48 B per particle, the pair rows)."""
    pair = 8 + 48 * springs
    return 2 * n * (88 + 24) + n * 288 + 2 * pairs * pair + 2 * bonds * 192 + (n * (24 + 8 + 16) + pairs * pair) / 5


def algorithmic_bytes_momentum(nf, nd, first):
    """Compulsory HBM bytes of one momentum launch: read each fluid particle's
    pos, vel, (rho, p, c, nu) once (3 x 32 B) and its list row count (4 B),
    each dummy's pos, vel, (c, nu, rho0), normal once (4 x 32 B); write the
    acceleration and the kicked velocity (2 x 32 B) and, in the first half,
    the drifted position (32 B).  Neighbour lists are an implementation aid
    and neighbour re-reads are cache traffic, so neither is counted."""
    return nf * (96 + 4 + 64 + (32 if first else 0)) + nd * 128


def max_over_ranks(torch, dist, ms, device):
    """The timed region's length as the slowest rank saw it (replicas: every
    rank times its own scene; the job is done when the last one is)."""
    if dist is None:
        return float(ms)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_step, steps, world, ms):
    """Whole-job throughput: the units all ranks processed / the max-over-ranks time."""
    return units_per_step * steps * world / (ms / 1e3)


def timed_steps(torch, solver, steps, flush):
    """Per-step CUDA-event times (ms) with an L2 flush before each step, outside
    the events."""
    times = []
    torch.cuda.synchronize()
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        solver.step(1)
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return times


def dem_case(torch, name, sc, steps, flush, peak, warm=20, block=10, what=""):
    """One DEM workload in mixed precision: `warm` steps (graph capture
    included), then `steps` steps timed `block` at a time with CUDA events,
    L2 flushed before each block; the roofline of the step against the
    per-step byte model with the measured pair and bond counts."""
    from this_studio_b200 import scenes

    s = scenes.build_dem(sc, "mixed")
    s.step(warm)
    ms = _event_steps(torch, s.step, steps, block, flush)
    n = int(sc.num_moving)
    pairs = int(s.getPairs(0)["objectPointed"].size)
    bonds = int(s.getBondedInteraction()["isBonded"].sum()) if sc.bonded else 0
    row = sc.hertz[0] if sc.hertz else None
    springs = 1 + (1 if row is not None and row[5] > 0 else 0) + (1 if row is not None and row[6] > 0 else 0)
    b = dem_bytes_8d(n, pairs, springs, bonds)
    achieved = b / (ms / 1e3) / 1e9
    d = s.diagnostics()
    return {"workload": name, "value": n / (ms / 1e3), "unit": METRIC, "ms_per_step": ms, "precision": "mixed",
            "steps": steps, "moving_particles": n, "pairs": pairs, "springs_per_pair": springs, "bonds": bonds,
            "what": what,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "algorithmic_bytes_per_step": b, "model": "dem_bytes_8d (bench.py)"},
            "diagnostics_fp64": {"momentum": [float(x) for x in d["momentum"]],
                                 "kinetic_energy": float(d["kineticEnergy"]),
                                 "rotational_energy": float(d["rotationalEnergy"])}}


def dem_cases(torch, flush, peak, stress):
    """The DEM rows: the plain bounce as specified (4,096 spheres, plane
    1 mm below the lowest nominal sphere bottom: few contacts), its
    contact-rich form (the same 4,096 spheres as a touching pack with
    friction, rolling and torsion), and the bonded beam + clumps."""
    from this_studio_b200 import scenes

    out = {"bounce": dem_case(torch, "dem_bounce_4096", scenes.dem_drop(), 200, flush, peak,
                              what="4,096 spheres: each kernel runs 4,096 threads, bound by the latency of their "
                                   "dependent loads"),
           "contact_rich": dem_case(torch, "dem_pack_4096", scenes.dem_pack(n_side=16), 200, flush, peak,
                                    what="the 4,096 spheres touching (1.1 (r_i + r_j) lists of ~11.5k pairs), "
                                         "friction, rolling and torsion springs")}
    if stress:
        out["beam_clumps"] = dem_case(torch, "bonded_beam_clumps_220k", scenes.bonded_beam_clumps(), 100, flush,
                                      peak, warm=10,
                                      what="20 x 20 x 400 bonded beam (462,840 bonds) + 20,000 three-sphere clumps")
    return out


def coupled_tank(torch, steps, warmup, flush):
    """Particle-level DEM-SPH coupling: eight DEM balls (r = 6 dx, densities
    500-2500) in a 64 x 64 x 48 tank of still water at dx = 0.01, two DEM
    substeps per fluid step, mixed precision; the same fluid stepped alone
    (markers held) for the coupling's overhead."""
    from this_studio_b200 import workloads

    sc = workloads.coupled_tank_scene()
    from this_studio_b200 import scenes

    f, d, c = scenes.build_coupled(sc, "mixed")
    c.step(max(warmup, 10), sc.dem_substeps)
    block = 10  # one captured block of coupled steps per timed call
    def run(fn):
        times = []
        torch.cuda.synchronize()
        for _ in range(max(1, steps // block)):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        return float(sum(times)) / (len(times) * block)
    ms = run(lambda: c.step(block, sc.dem_substeps))
    ms_fluid = run(lambda: f.step(block))
    nm, nb = c.numMarkers()
    nf = sc.sph.fluid.shape[0]
    return {"workload": "coupled_tank_200k", "value": nf / (ms / 1e3), "unit": METRIC, "ms_per_step": ms,
            "fluid_alone_ms_per_step": ms_fluid, "fluid_particles": nf, "dummy_particles": sc.sph.dummy.shape[0],
            "balls": nb, "markers": nm, "dem_substeps": sc.dem_substeps, "precision": "mixed", "steps": steps}


def ice_sheet(torch, steps):
    """The coupled ice-sheet stress scene: about 1M bonded r = 2 mm spheres
    moving into a 20,000-triangle cylinder, floating on 2M WCSPH particles
    (dx = 4 mm, 3M floor dummies), coupled particle by particle (one marker per
    ball), one DEM step per fluid step, mixed precision.  Particles counted:
    balls + fluid."""
    from this_studio_b200 import scenes

    sc = scenes.ice_sheet_on_water()
    f, d, c = scenes.build_coupled(sc, "mixed")
    c.step(10, sc.dem_substeps)
    n = sc.dem.position.shape[0] + sc.sph.fluid.shape[0]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    c.step(steps, sc.dem_substeps)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    nm, nb = c.numMarkers()
    return {"workload": "ice_sheet_coupled_3m", "value": n / (ms / 1e3), "unit": METRIC, "ms_per_step": ms,
            "balls": int(sc.dem.position.shape[0]), "fluid_particles": int(sc.sph.fluid.shape[0]),
            "dummy_particles": int(sc.sph.dummy.shape[0]), "markers": nm, "triangles": 20000,
            "dem_substeps": sc.dem_substeps, "precision": "mixed", "steps": steps}


def served_stream(torch, num, seed=5, rate=100.0, steps=500, chunk=100, fp64_sample=200, warm=True):
    """The serving / batching stream: `num` seeded scenes (DEM drops and WCSPH
    dam breaks, particle counts log-uniform over 1k-200k, polydisperse DEM
    radii with sigma 0.2 and max/min <= 3, 500 steps each) arriving as a
    Poisson process at `rate` per second -- an offered load above the
    server's capacity, so the queue builds and the throughput is the
    server's -- served by the continuous-batching server in mixed precision
    (batches of up to 512 members, admitted by an HBM budget); then the same
    scenes one after another on the plain solver in mixed precision, and the
    first `fp64_sample` of them in FP64.  Wall-clock times; scenes are
    generated before each clock starts."""
    from this_studio_b200 import serve

    n_max = 200_000
    c0, dt = serve.stream_params(n_max)
    mk = lambda k: serve.make_stream(k, seed=seed, n_min=1000, n_max=n_max, rate=rate, steps=steps)
    # warm-up on a stream of the same sizes (another seed): kernel loads, graph
    # executables and the memory pool grown to the stream's working set, as in
    # a server that has been running; the autotuner (cell size, list shape,
    # skin, capacities per kind) runs on that warm-up stream's scenes
    tunings, tune = None, None
    if warm:
        w = serve.SceneServer(hbm_budget=55e9, chunk=chunk, precision="mixed", sph_c0=c0, sph_dt=dt, autotune=True)
        wm = w.run(serve.make_stream(24, seed=1, n_min=1000, n_max=n_max, rate=1e3, steps=100))
        tunings, tune = w.tunings, {"seconds": wm.get("tune_s"), **wm.get("tuning", {})}
    reqs = mk(num)
    ps = serve.particle_steps(reqs, c0, dt)
    n_dem = sum(1 for r in reqs if r.kind == "dem")
    srv = serve.SceneServer(hbm_budget=55e9, chunk=chunk, precision="mixed", max_members=512, sph_c0=c0, sph_dt=dt,
                            tunings=tunings)
    torch.cuda.synchronize()
    m = srv.run(reqs)
    del reqs
    plain_kind = {}
    plain_mixed = ps / serve.run_plain(mk(num), "mixed", c0, dt, per_kind=plain_kind)
    # each kind's throughput on its own: served = its particle-steps over the
    # time its batch was stepping (the kinds overlap on the device), plain =
    # over its scenes' time on the plain solver
    kinds = {}
    for k, (sec, kps) in plain_kind.items():
        pk = m["per_kind"].get(k, {})
        served_k = pk.get("particle_steps", 0) / pk["busy_s"] if pk.get("busy_s") else None
        kinds[k] = {"particle_steps": kps, "plain_s": sec, "plain_value": kps / sec,
                    "served_busy_value": served_k,
                    "served_busy_vs_plain": None if served_k is None else served_k / (kps / sec)}
    k = min(fp64_sample, num)
    sample = mk(k)
    ps_k = serve.particle_steps(sample, c0, dt)
    plain_fp64 = ps_k / serve.run_plain(sample, "fp64", c0, dt)
    return {"workload": f"served_stream_{num}", "scenes": num, "dem_scenes": n_dem, "seed": seed,
            "arrival_rate_per_s": rate, "steps_per_scene": steps, "chunk_steps": chunk, "max_members": 512,
            "particle_steps": ps, "value": m["value"], "unit": METRIC, "makespan_s": m["makespan_s"],
            "plain_mixed_value": plain_mixed, "speedup_vs_plain_mixed": m["value"] / plain_mixed,
            "plain_fp64_value": plain_fp64, "plain_fp64_what": f"the first {k} scenes of the stream",
            "speedup_vs_plain_fp64": m["value"] / plain_fp64,
            "scene_step_latency_p50_ms": m["scene_step_latency_p50_ms"],
            "scene_step_latency_p99_ms": m["scene_step_latency_p99_ms"],
            "scene_latency_p50_s": m["scene_latency_p50_s"], "scene_latency_p99_s": m["scene_latency_p99_s"],
            "admission_wait_p50_s": m["admission_wait_p50_s"], "admission_wait_p99_s": m["admission_wait_p99_s"],
            "per_kind": m["per_kind"], "per_kind_vs_plain": kinds, "autotune": tune}


def pipeline_traffic(tj):
    """DRAM bytes per launch of the momentum kernel inside the step (caches as
    the step leaves them, L2 flushed between steps): first and second pass
    from profiles/traffic.json, or None."""
    p = tj.get("in_pipeline")
    if not p:
        return None
    a, b = p["k_sph_accel_u_first_pass"], p["k_sph_accel_u_second_pass"]
    return {"first_pass": a["dram_read"] + a["dram_write"], "second_pass": b["dram_read"] + b["dram_write"],
            "first_pass_note": a.get("note"), "source": "profiles/traffic.json in_pipeline"}


def native(args, rank, world, dist):
    import torch

    import this_studio_b200 as tsb
    from this_studio_b200 import _lib
    from this_studio_b200.scenes import build_sph

    torch.cuda.set_device(rank % max(1, torch.cuda.device_count()))
    dev = torch.device("cuda", torch.cuda.current_device())
    sc = workload()
    nf, nd = sc.fluid.shape[0], sc.dummy.shape[0]
    solver = build_sph(sc, args.precision)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    peaks = {}
    pk_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk_path):
        peaks = json.load(open(pk_path))
    peak = peaks.get("hbm_gbs", 6650.0)
    # warm-up: the requested steps, then single steps so that the one-step
    # graphs of both buffer states are captured before the timed region
    solver.step(max(args.warmup, 3))
    for _ in range(4):
        solver.step(1)
    torch.cuda.synchronize()
    diag0 = solver.diagnostics()
    if dist:
        dist.barrier()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    launches0 = tsb.kernel_launches()
    rebuilds0 = solver.skinStats()[1]
    times = timed_steps(torch, solver, args.steps, flush)
    torch.cuda.synchronize()
    # the launch counter sees host-issued launches; a list rebuild inside a
    # graph step is a conditional node whose kernels run only when the
    # device decides to rebuild: add them per rebuild
    cond_active, per_rebuild = solver.conditionalRebuild()
    rebuilds = solver.skinStats()[1] - rebuilds0
    launches = tsb.kernel_launches() - launches0 + (rebuilds * per_rebuild if cond_active else 0)
    clk = clocks.stop()
    diag1 = solver.diagnostics()
    total_ms = float(sum(times))
    total_ms = max_over_ranks(torch, dist, total_ms, dev)
    value = replica_value(nf, args.steps, world, total_ms)
    step_ms = total_ms / args.steps

    # per-kernel live timing for the roofline (same stream, events per phase)
    import ctypes as C

    phases = (C.c_double * 5)()
    nprof = min(args.steps, 20)
    _lib.call("demsph_sph_profile_steps", solver._h, nprof, phases)
    ph = list(phases)
    mom_ms = 0.5 * (ph[2] + ph[4])
    impl_bytes = 0.5 * (algorithmic_bytes_momentum(nf, nd, True) + algorithmic_bytes_momentum(nf, nd, False))
    mom_bytes = momentum_bytes_8d(nf, nd)
    achieved = mom_bytes / (mom_ms / 1e3) / 1e9
    ncell = 1
    for a, b in zip(sc.minb, sc.maxb):
        ncell *= max(1, int((b - a) / (2.0 * 1.3 * sc.spacing * 1.04)))
    step_bytes = sph_bytes_8d(nf, nd, ncell)
    tj = {}
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        tj = json.load(open(tpath))
    traffic = tj.get("k_sph_accel_bytes_per_launch")
    inst = tj.get("k_sph_accel_warp_instructions_per_launch")
    flop = tj.get("k_sph_accel_fp32_flop_per_launch")
    sm_hz = (clk.get("sm_mhz") or 1965.0) * 1e6

    # end to end through the public API: upload, K steps, read back.  Three
    # complete runs (each scene destroyed after its read-back), the median
    # reported: the first one also pays for mapping fresh device memory, which
    # on a shared GPU has varied from 10 ms to 300 ms; the later ones reuse
    # the memory the library's pool keeps (its default).  Each run's time is
    # split by host timers into scene set-up (add + initialise), the steps and
    # the read-back.
    runs_s, parts = [], []
    for _ in range(3):
        torch.cuda.synchronize()
        h0 = time.perf_counter()
        s2 = build_sph(sc, args.precision)
        torch.cuda.synchronize()
        h1 = time.perf_counter()
        s2.step(args.steps)
        torch.cuda.synchronize()
        h2 = time.perf_counter()
        out = s2.getSPH()
        torch.cuda.synchronize()
        h3 = time.perf_counter()
        runs_s.append(h3 - h0)
        parts.append({"setup_ms": 1e3 * (h1 - h0), "steps_ms": 1e3 * (h2 - h1), "readback_ms": 1e3 * (h3 - h2)})
        del s2
        torch.cuda.synchronize()
    k = sorted(range(3), key=lambda i: runs_s[i])[1]
    e2e_s = runs_s[k]
    h2d = (nf + nd) * (3 * 8 * 2 + 4 * 8)  # positions, velocities, 4 scalars per particle
    d2h = sum(v.nbytes for v in out.values()) + 16 * args.steps  # final state + per-step status word
    e2e = nf * args.steps * world / e2e_s

    # the other precision and the DEM workloads, next to the headline
    other = "fp64" if args.precision == "mixed" else "mixed"
    s3 = build_sph(sc, other)
    s3.step(3)
    for _ in range(4):
        s3.step(1)
    t3 = timed_steps(torch, s3, min(args.steps, 100), flush)
    del s3
    other_value = nf / (float(sum(t3)) / len(t3) / 1e3)
    dem = dem_cases(torch, flush, peak, args.stress)
    coupled = coupled_tank(torch, 100, args.warmup, flush)
    del flush
    ice = ice_sheet(torch, 40) if args.stress else None
    stream = served_stream(torch, args.stream) if (args.stream > 0 and rank == 0 and world == 1) else None

    fp32_peak = 148 * 128 * 2 * sm_hz
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32",
        "data": "synthetic (seeded lattice dam break, no dataset)",
        "config": {"workload": WORKLOAD, "fluid_particles": nf, "dummy_particles": nd, "h": 1.3 * sc.spacing,
                   "dt": sc.dt, "precision": args.precision,
                   "precision_note": "FP32 force arithmetic, FP64 positions / velocities / density accumulation"
                   if args.precision == "mixed" else "FP64 throughout (the reference's arithmetic)",
                   "l2": "flushed (256 MB write) between timed steps", "parallelism": f"replicas x{world}"},
        "value_" + other: other_value,
        "dem": dem,
        "coupled": coupled,
        "ice_sheet": ice,
        "stream": stream,
        "gpu_launches": int(launches),
        "list_rebuilds": {"timed_steps": int(rebuilds), "conditional_graph_node": bool(cond_active),
                          "kernels_per_rebuild": int(per_rebuild)},
        "clocks": clk,
        "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": h2d / args.steps,
                "d2h_bytes_per_step": d2h / args.steps,
                "what": "build scene from host arrays, initialise, K steps, read state back; median of 3 runs",
                "runs_s": runs_s, "first_run_value": nf * args.steps * world / runs_s[0],
                "median_run_parts_ms": parts[k], "setup_ms_per_scene": parts[k]["setup_ms"],
                "readback_ms_per_scene": parts[k]["readback_ms"]},
        # the dominant kernel against the compulsory bytes of one momentum
        # pass of the mixed-precision design (72 B read + 12 B written per
        # fluid particle, 24 B per dummy); the step against the per-step model
        "roofline": {"bound": "hbm", "kernel": "k_sph_accel_u", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "traffic_what": "cold L2 per launch (ncu flushes before each profiled launch)",
                     "traffic_in_pipeline": pipeline_traffic(tj),
                     "algorithmic_bytes_per_launch": mom_bytes, "ms_per_launch": mom_ms,
                     "model": "momentum_bytes_8d (bench.py)",
                     "implementation_bytes_per_launch": impl_bytes,
                     "implementation_frac": impl_bytes / (mom_ms / 1e3) / 1e9 / peak,
                     "step": {"algorithmic_bytes": step_bytes, "achieved": step_bytes / (step_ms / 1e3) / 1e9,
                              "frac": step_bytes / (step_ms / 1e3) / 1e9 / peak},
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback 6650 GB/s"},
        # the bounds the SPH passes actually sit at: FP32 SIMT throughput and
        # warp-instruction issue (4 per SM per clock; 148 SMs at the sampled
        # SM clock); flop and instruction counts per launch from the committed
        # ncu capture, time live
        "fp32_simt": None if not flop else {
            "kernel": "k_sph_accel_u", "achieved": flop / (mom_ms / 1e3) / 1e12, "unit": "TFLOP/s",
            "peak": fp32_peak / 1e12, "frac": flop / (mom_ms / 1e3) / fp32_peak, "flop_per_launch": flop,
            "source": "profiles/traffic.json (ncu: 2 x ffma + fadd + fmul thread instructions)"},
        "issue_roofline": None if not inst else {
            "kernel": "k_sph_accel_u", "achieved": inst / (mom_ms / 1e3), "unit": "warp-instructions/s",
            "peak": 4 * 148 * sm_hz, "frac": inst / (mom_ms / 1e3) / (4 * 148 * sm_hz),
            "instructions_per_launch": inst, "source": "profiles/traffic.json (ncu smsp__inst_executed.sum)"},
        "phase_ms": {"cell_sort": ph[0], "reorder_lists": ph[1], "momentum_1": ph[2], "continuity_eos": ph[3],
                     "momentum_2": ph[4]},
        "conservation_fp64": {
            "what": "device diagnostics of the fluid before and after the timed steps",
            "mass_change": diag1["mass"] - diag0["mass"],
            "momentum_before": [float(x) for x in diag0["momentum"]],
            "momentum_after": [float(x) for x in diag1["momentum"]],
            "kinetic_energy": [diag0["kineticEnergy"], diag1["kineticEnergy"]],
            "potential_energy": [diag0["potentialEnergy"], diag1["potentialEnergy"]],
            "density_change_sum": [diag0["densityChangeSum"], diag1["densityChangeSum"]]},
    }
    if rank == 0:
        line["cpu_baseline"] = cpu_baseline(sc)
        if world == 1:
            fl = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
            mine = {"sph": step_ms, "dem": dem["bounce"]["ms_per_step"],
                    "beam": beam_only(torch, 20, fl) if args.stress else None}
            line["reference_cuda"] = reference_cuda_baseline(torch, sc, min(args.steps, 50), args.warmup, fl, mine)
            del fl
    return line


def _event_steps(torch, fn, steps, block, flush):
    """Mean ms per step of `steps` steps run `block` at a time, each block
    bracketed by CUDA events on the current stream, L2 flushed before it."""
    times = []
    torch.cuda.synchronize()
    for _ in range(max(1, steps // block)):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn(block)
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return float(sum(times)) / (len(times) * block)


def reference_cuda_baseline(torch, sc, steps, warmup, flush, mine_ms):
    """Baseline leg: the reference's own CUDA kernels (DEMSPH/kernel/*.cu built
    from its sources for sm_100a with its Release flags, oracle/Makefile.ref)
    driven as its solvers drive them (oracle/ref_harness: WCSPHSolver::solve's
    step, DEMSolver's loop_ball_wall), FP64 as the reference computes, on the
    same workloads as this library's lines, same L2 flush, CUDA events.  The
    reference reads its pair counts back to the host in every neighbour
    search, as its solvers do; that is part of its step.  DEM rows: the
    4,096-sphere bounce and the bonded beam without the clumps (the
    reference's clump force gather reads past its clump array,
    ballIntegrationKernel.cu:20, so clumps are not run on it)."""
    from oracle import ref_harness
    from this_studio_b200 import scenes

    if not ref_harness.available():
        return {"unavailable": "oracle/_ref/libdemsph_ref.so not built (no reference checkout at build time)"}
    out = {"what": "the reference's CUDA kernels built from its sources (sm_100a, -O3), FP64, its launch geometry"}
    r = ref_harness.RefSPH(sc, torch)
    r.step(max(warmup, 3))
    ms = _event_steps(torch, r.step, steps, 1, flush)
    nf = sc.fluid.shape[0]
    out["sph"] = {"workload": WORKLOAD, "ms_per_step": ms, "value": nf / (ms / 1e3), "unit": METRIC,
                  "this_library_ms_per_step": mine_ms["sph"], "speedup": ms / mine_ms["sph"]}
    del r
    dem = scenes.dem_drop()
    r = ref_harness.RefDEM(dem, torch)
    r.initialize()
    r.step(max(warmup, 5))
    ms = _event_steps(torch, r.step, min(steps * 5, 200), 10, flush)
    out["dem_bounce"] = {"workload": "dem_bounce_4096", "ms_per_step": ms, "value": 4096 / (ms / 1e3),
                         "unit": METRIC, "this_library_ms_per_step": mine_ms["dem"],
                         "speedup": ms / mine_ms["dem"]}
    del r
    if mine_ms.get("beam") is not None:
        beam = scenes.bonded_beam_clumps(n_clumps=0)
        r = ref_harness.RefDEM(beam, torch)
        r.initialize()
        r.step(5)
        ms = _event_steps(torch, r.step, min(steps, 20), 5, flush)
        nmov = int((~beam.fixed).sum())
        out["bonded_beam"] = {"workload": "bonded_beam_160k", "ms_per_step": ms, "value": nmov / (ms / 1e3),
                              "unit": METRIC, "bonds": r.nb, "this_library_ms_per_step": mine_ms["beam"],
                              "speedup": ms / mine_ms["beam"]}
        del r
    torch.cuda.empty_cache()
    return out


def beam_only(torch, steps, flush):
    """The bonded beam of the beam + clumps scene alone (160,000 spheres, the
    x = 0 layer clamped, 462,840 bonds), the workload the reference's own
    kernels are timed on; mixed precision."""
    from this_studio_b200 import scenes

    sc = scenes.bonded_beam_clumps(n_clumps=0)
    s = scenes.build_dem(sc, "mixed")
    s.step(5)
    return _event_steps(torch, s.step, steps, 5, flush)


def cpu_baseline(sc, steps=2):
    """The FP64 C++ oracle (the reference's step restated; OpenMP) on the host
    cores, a bounded sample of the same workload."""
    from oracle import oracle

    oracle.build()
    threads = oracle.set_threads(os.cpu_count() or 1)
    o = oracle.OracleSPH()
    o.add_sph(sc.fluid, None, sc.sound_speed, sc.spacing, sc.density, sc.viscosity)
    o.add_dummy(sc.dummy, None, sc.sound_speed, sc.spacing, sc.density, sc.viscosity)
    o.initialize(sc.minb, sc.maxb, sc.gravity, sc.dt)
    o.step(1)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    return {"value": sc.fluid.shape[0] * steps / dt, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{steps} steps of the full {sc.fluid.shape[0]}-particle workload after 1 warm-up step"}


def reference(args, rank, world):
    if rank != 0:
        return None
    from oracle import oracle

    sc = workload()
    oracle.build()
    threads = oracle.set_threads(os.cpu_count() or 1)
    o = oracle.OracleSPH()
    o.add_sph(sc.fluid, None, sc.sound_speed, sc.spacing, sc.density, sc.viscosity)
    o.add_dummy(sc.dummy, None, sc.sound_speed, sc.spacing, sc.density, sc.viscosity)
    o.initialize(sc.minb, sc.maxb, sc.gravity, sc.dt)
    # each step of this arm is the full workload step; bound the sample so the
    # run ends within minutes on a many-core host
    steps = max(1, min(args.steps, 5))
    warm = max(1, min(args.warmup, 1))
    o.step(warm)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    v = sc.fluid.shape[0] * steps / dt
    return {"metric": METRIC, "value": v, "unit": METRIC, "impl": "reference", "n_gpus": world, "steps": steps,
            "warmup": warm, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lattice dam break, no dataset)",
            "config": {"workload": WORKLOAD, "fluid_particles": sc.fluid.shape[0],
                       "dummy_particles": sc.dummy.shape[0]},
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": threads, "kind": "port",
                             "sample": f"{steps} full steps after {warm} warm-up step(s)"},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist

        backend = "gloo" if args.impl == "reference" else "nccl"
        tdist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        dist = tdist
    try:
        if args.impl == "reference":
            line = reference(args, rank, world)
        else:
            line = native(args, rank, world, dist)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
