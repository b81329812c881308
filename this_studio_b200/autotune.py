"""The autotuner: cell size, list-build block shape, skin and list capacity
for a kind of scene, chosen by timing steps of a representative scene on the
device.

The reference fixes these by hand: the ball grid's cell is 2 r_max
(DEMSolver.h:245-263), the SPH cell 2 h_max (WCSPHSolver.h:119-150), the
block size 256 (DEMSolver.h:149) and the pair capacities 6 N and 80 N
(DEMSolver.h:174, WCSPHSolver.h:119).  Here each candidate cell factor (the
cell edge as a multiple of the reference's) builds the scene afresh and times
`steps` steps after `warmup` with CUDA events on the scene's stream; the
fastest is kept.  On the chosen build the SPH list-build block shape and skin
are tuned in place (demsph_sph_tune, demsph_sph_tune_skin).  Capacities come
from demand: the DEM pair / reverse / triangle rows per ball and the SPH row
headroom are set to what the timed run grew them to, so scenes of the same
kind built with the tuning do not overflow and replay steps.

A candidate replaces the default (factor 1, shape 0, the grid's skin) only
when it is faster by more than `margin` (5%): timings of a short run differ
by a few percent from run to run, and a setting picked on noise costs more on
the large scenes that carry a stream than it saves on the small one it was
timed on.

Every choice gives the same pairs; a different cell size orders rows
differently, so sums differ by rounding.  A Tuning applies to later scenes
through `configure` (before initialisation) and `finish` (after it); the
batched and served forms take one per kind."""
from __future__ import annotations

from dataclasses import asdict, dataclass, field

from . import scenes as S

DEM_FACTORS = (1.0, 1.25, 1.5)
SPH_FACTORS = (1.0, 1.15, 1.3)
MARGIN = 0.05


def _pick(default, ms, margin):
    """The fastest key of ms if it beats ms[default] by more than `margin`, else default."""
    best = min(ms, key=ms.get)
    return best if ms[best] < (1.0 - margin) * ms[default] else default


@dataclass
class Tuning:
    kind: str                              # "dem" or "sph"
    cell_factor: float = 1.0
    reserve: tuple = None                  # DEM: (pairs, reverse, triangles) per ball
    list_shape: int = None                 # SPH: list-build block shape index
    skin: float = None                     # SPH: skin fraction
    headroom: float = None                 # SPH: row capacity above the initial longest row
    ms_per_step: dict = field(default_factory=dict)   # cell factor -> ms per step
    ms_per_shape: list = None              # SPH: ms per list build of each shape
    ms_per_skin: list = None               # SPH: ms per step with no, half and full skin

    def configure(self, solver):
        """Settings applied before initialisation."""
        solver.setCellFactor(self.cell_factor)
        if self.kind == "dem":
            if self.reserve is not None:
                solver.reserve(*self.reserve)
        elif self.headroom is not None:
            solver.setListHeadroom(self.headroom)

    def finish(self, solver):
        """Settings applied after initialisation."""
        if self.kind == "sph":
            if self.list_shape is not None:
                solver.setListShape(self.list_shape)
            if self.skin is not None:
                solver.setSkin(self.skin)  # at most the grid's skin: the candidates were no, half and full

    def as_dict(self):
        d = asdict(self)
        d["ms_per_step"] = {str(k): v for k, v in self.ms_per_step.items()}
        return d


def _ms_per_step(torch, solver, stream, steps, warmup):
    solver.step(warmup)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    solver.step(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def tune_dem(scene, precision="mixed", factors=DEM_FACTORS, steps=50, warmup=10, margin=MARGIN):
    """Tuning for DEM scenes like `scene` (cell factor and row capacities)."""
    import torch

    stream = torch.cuda.Stream()
    t = Tuning("dem")
    caps = {}
    for f in factors:
        s = S.build_dem(scene, precision, stream, configure=lambda x, f=f: x.setCellFactor(f))
        t.ms_per_step[f] = _ms_per_step(torch, s, stream, steps, warmup)
        caps[f] = s.capacity()
        del s
    t.cell_factor = _pick(factors[0], t.ms_per_step, margin)
    t.reserve = caps[t.cell_factor]
    return t


def tune_sph(scene, precision="mixed", factors=SPH_FACTORS, steps=40, warmup=6, trials=3, margin=MARGIN):
    """Tuning for WCSPH scenes like `scene` (cell factor, list-build block
    shape, skin, row headroom)."""
    import torch

    stream = torch.cuda.Stream()
    t = Tuning("sph")
    for f in factors:
        s = S.build_sph(scene, precision, stream, configure=lambda x, f=f: x.setCellFactor(f))
        t.ms_per_step[f] = _ms_per_step(torch, s, stream, steps, warmup)
        del s
    t.cell_factor = best = _pick(factors[0], t.ms_per_step, margin)
    s = S.build_sph(scene, precision, stream, configure=lambda x: x.setCellFactor(best))
    cap0 = s.listCapacity()
    skin0 = s.skinStats()[0]
    s.step(warmup)
    _, ms_shape = s.tune(trials)
    t.ms_per_shape = [float(x) for x in ms_shape]
    t.list_shape = _pick(0, dict(enumerate(t.ms_per_shape)), margin)
    s.setListShape(t.list_shape)
    _, ms_skin = s.tuneSkin(steps)  # no skin, half and all of the grid's skin
    t.ms_per_skin = [float(x) for x in ms_skin]
    t.skin = (0.0, 0.5 * skin0, skin0)[_pick(2, dict(enumerate(t.ms_per_skin)), margin)]
    s.setSkin(t.skin)
    s.step(steps)
    cap1 = s.listCapacity()
    # initial rows were (1 + 1/8) x the longest; cover the growth seen since
    grow = max(c1 / c0 for c0, c1 in zip(cap0, cap1) if c0 > 0)
    t.headroom = float(min(4.0, (1.0 + 0.125) * grow - 1.0))
    del s
    return t
