"""Batched form: many independent scenes stepped as one device scene.

Each member scene is translated into its own tile of the x-y plane; tiles are
separated by empty cells, so no pair crosses between members and every
member's grid neighbourhood is its own.  The physics is translation
invariant and the cell (>= 2 r_max, >= 2 h_max) still contains every
interacting pair, so a member evolves as it does alone, up to rounding of the
translated coordinates, while all members share one set of kernel launches
per step (one cell sort, one pair pass, one reduction, ...).

Membership changes (admission, retirement) rebuild the device scene at a
step boundary and carry each continuing member's state across: positions,
velocities and angular velocities, ball-ball and ball-wall springs (DEM), and
density / pressure / density change (SPH).  DEM members change only at steps
that are multiples of 5, the reference's re-sort cadence (DEMSolver.h:1384),
so the pair list is rebuilt on the same steps as when the member runs alone.

Members keep the reference's domain-edge behaviour only while their particles
stay inside their own domain box: a particle that leaves it is clamped into
the edge cells of the batch domain rather than of its own.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import scenes as S


@dataclass
class Member:
    key: int
    scene: object
    offset: np.ndarray = None
    steps_done: int = 0
    # carried state (member-local coordinates / indices)
    state: dict = field(default_factory=dict)


def tile_offsets(boxes, gap):
    """Shelf-packs axis-aligned boxes (lo, hi) into rows along x, rows stacked
    along y, all at their own z.  Returns one translation per box."""
    sizes = [np.asarray(hi, float) - np.asarray(lo, float) for lo, hi in boxes]
    total = sum(s[0] * s[1] for s in sizes)
    row_w = max(max(s[0] for s in sizes), math.sqrt(total)) + gap
    offs = []
    x = y = row_h = 0.0
    for (lo, hi), sz in zip(boxes, sizes):
        if x > 0 and x + sz[0] > row_w:
            x = 0.0
            y += row_h + gap
            row_h = 0.0
        offs.append(np.array([x - lo[0], y - lo[1], 0.0]))
        x += sz[0] + gap
        row_h = max(row_h, sz[1])
    return offs


class DEMBatch:
    """DEM members of one time step and gravity stepped together."""

    def __init__(self, precision="mixed", stream=None):
        self.precision = precision
        self.stream = stream
        self.members: list[Member] = []
        self.solver = None
        self.ranges = []

    @staticmethod
    def cell_of(scene):
        return 2.0 * float(np.max(scene.radius))

    def _materials(self):
        """One material id per distinct material row set; members that share
        parameters share ids."""
        sig = {}
        ids = []
        rows_h, rows_l, rows_b = [], [], []
        for m in self.members:
            key = (tuple(map(tuple, m.scene.hertz)), tuple(map(tuple, m.scene.linear)),
                   tuple(map(tuple, m.scene.bonded)))
            if key not in sig:
                mats = sorted({int(v) for v in m.scene.material} |
                              {int(w["material"]) for w in m.scene.walls} |
                              {int(r[i]) for r in m.scene.hertz + m.scene.linear + m.scene.bonded for i in (0, 1)})
                base = sum(len(v[1]) for v in sig.values())
                remap = {mid: base + k for k, mid in enumerate(mats)}
                sig[key] = (remap, mats)
                for r in m.scene.hertz:
                    rows_h.append((remap[int(r[0])], remap[int(r[1])]) + tuple(r[2:]))
                for r in m.scene.linear:
                    rows_l.append((remap[int(r[0])], remap[int(r[1])]) + tuple(r[2:]))
                for r in m.scene.bonded:
                    rows_b.append((remap[int(r[0])], remap[int(r[1])]) + tuple(r[2:]))
            ids.append(sig[key][0])
        return ids, rows_h, rows_l, rows_b

    def rebuild(self):
        """(Re)creates the device scene from the members' current states."""
        from .scenes import DEMScene

        self.solver = None
        if not self.members:
            return
        cell = max(self.cell_of(m.scene) for m in self.members)
        boxes = [(np.asarray(m.scene.minb), np.asarray(m.scene.maxb)) for m in self.members]
        offs = tile_offsets(boxes, gap=2.0 * cell)
        remaps, rows_h, rows_l, rows_b = self._materials()
        pos, vel, w, rad, den, mat, fixed = [], [], [], [], [], [], []
        walls = []
        lo = np.full(3, np.inf)
        hi = np.full(3, -np.inf)
        self.ranges = []
        self.tri_ranges = []
        start = 0
        tstart = 0
        for m, off, remap in zip(self.members, offs, remaps):
            sc = m.scene
            m.offset = off
            st = m.state
            n = sc.position.shape[0]
            pos.append((st["position"] if "position" in st else sc.position) + off)
            v0 = sc.velocity if sc.velocity is not None else np.zeros((n, 3))
            w0 = getattr(sc, "angvel", None)
            w0 = w0 if w0 is not None else np.zeros((n, 3))
            vel.append(st.get("velocity", v0))
            w.append(st.get("angularVelocity", w0))
            rad.append(sc.radius)
            den.append(sc.density)
            mat.append(np.array([remap[int(x)] for x in sc.material], np.int32))
            fixed.append(np.zeros(n, bool) if sc.fixed is None else sc.fixed)
            for wl in sc.walls:
                d = dict(wl)
                d["position"] = np.asarray(wl["position"], float) + off
                d["material"] = remap[int(wl["material"])]
                walls.append(d)
            nt = sum(len(wl["tri0"]) for wl in sc.walls)
            self.ranges.append((start, start + n))
            self.tri_ranges.append((tstart, tstart + nt))
            start += n
            tstart += nt
            lo = np.minimum(lo, np.asarray(sc.minb) + off)
            hi = np.maximum(hi, np.asarray(sc.maxb) + off)
        first = self.members[0].scene
        big = DEMScene(name="batch", position=np.concatenate(pos), radius=np.concatenate(rad),
                       density=np.concatenate(den), material=np.concatenate(mat),
                       velocity=np.concatenate(vel), fixed=np.concatenate(fixed), hertz=rows_h, linear=rows_l,
                       bonded=rows_b, walls=walls, minb=tuple(lo), maxb=tuple(hi), gravity=first.gravity,
                       dt=first.dt)
        big.angvel = np.concatenate(w)
        self.solver = S.build_dem(big, self.precision, self.stream)
        # contact history of continuing members, renumbered into the batch
        A, B, SL, RO, TO = [], [], [], [], []
        WA, WT, WS, WR, WTo = [], [], [], [], []
        for m, (b0, _), (t0, _) in zip(self.members, self.ranges, self.tri_ranges):
            st = m.state
            if "pairs" in st:
                p = st["pairs"]
                A.append(p["a"] + b0); B.append(p["b"] + b0)
                SL.append(p["sliding"]); RO.append(p["rolling"]); TO.append(p["torsion"])
            if "wall_pairs" in st:
                p = st["wall_pairs"]
                WA.append(p["a"] + b0); WT.append(p["b"] + t0)
                WS.append(p["sliding"]); WR.append(p["rolling"]); WTo.append(p["torsion"])
        if A:
            self.solver.importSprings(np.concatenate(A), np.concatenate(B), np.concatenate(SL), np.concatenate(RO),
                                      np.concatenate(TO))
        if WA:
            self.solver.importWallSprings(np.concatenate(WA), np.concatenate(WT), np.concatenate(WS),
                                          np.concatenate(WR), np.concatenate(WTo))

    def capture(self):
        """Copies every member's state out of the device scene."""
        if self.solver is None:
            return
        b = self.solver.getBall()
        pp = self.solver.getPairs(0)
        wp = self.solver.getPairs(1)
        for m, (b0, b1), (t0, t1) in zip(self.members, self.ranges, self.tri_ranges):
            st = m.state
            st["position"] = b["position"][b0:b1] - m.offset
            st["velocity"] = b["velocity"][b0:b1]
            st["angularVelocity"] = b["angularVelocity"][b0:b1]
            sel = (pp["objectPointed"] >= b0) & (pp["objectPointed"] < b1)
            st["pairs"] = {"a": pp["objectPointed"][sel] - b0, "b": pp["objectPointing"][sel] - b0,
                           "sliding": pp["sliding"][sel], "rolling": pp["rolling"][sel],
                           "torsion": pp["torsion"][sel]}
            sel = (wp["objectPointed"] >= b0) & (wp["objectPointed"] < b1)
            st["wall_pairs"] = {"a": wp["objectPointed"][sel] - b0, "b": wp["objectPointing"][sel] - t0,
                                "sliding": wp["sliding"][sel], "rolling": wp["rolling"][sel],
                                "torsion": wp["torsion"][sel]}

    def step(self, n):
        if self.solver is not None and n > 0:
            self.solver.step(n)
            for m in self.members:
                m.steps_done += n

    def num_particles(self):
        return sum(m.scene.num_moving for m in self.members)


class SPHBatch:
    """WCSPH members of one time step and gravity stepped together."""

    def __init__(self, precision="mixed", stream=None):
        self.precision = precision
        self.stream = stream
        self.members: list[Member] = []
        self.solver = None
        self.ranges = []

    def rebuild(self):
        from .solvers import WCSPHSolver

        self.solver = None
        if not self.members:
            return
        cell = max(2.0 * 1.3 * m.scene.spacing for m in self.members)
        boxes = [(np.asarray(m.scene.minb), np.asarray(m.scene.maxb)) for m in self.members]
        offs = tile_offsets(boxes, gap=2.0 * cell)
        s = WCSPHSolver(self.stream)
        lo = np.full(3, np.inf)
        hi = np.full(3, -np.inf)
        self.ranges = []
        start = 0
        for m, off in zip(self.members, offs):
            sc = m.scene
            m.offset = off
            n = sc.fluid.shape[0]
            s.addSPHs(m.state.get("position", sc.fluid) + off, m.state.get("velocity"), sc.sound_speed, sc.spacing,
                      sc.density, sc.viscosity)
            self.ranges.append((start, start + n))
            start += n
            lo = np.minimum(lo, np.asarray(sc.minb) + off)
            hi = np.maximum(hi, np.asarray(sc.maxb) + off)
        for m, off in zip(self.members, offs):
            sc = m.scene
            s.addDummies(sc.dummy + off, None, sc.sound_speed, sc.spacing, sc.density, sc.viscosity)
        first = self.members[0].scene
        s.initialize(tuple(lo), tuple(hi), first.gravity, first.dt, self.precision)
        if any("density" in m.state for m in self.members):
            n = start
            rho = np.empty(n)
            p = np.empty(n)
            dr = np.empty(n)
            for m, (a, b) in zip(self.members, self.ranges):
                rho[a:b] = m.state.get("density", np.full(b - a, m.scene.density))
                p[a:b] = m.state.get("pressure", np.zeros(b - a))
                dr[a:b] = m.state.get("densityChange", np.zeros(b - a))
            s.setSPH(density=rho, pressure=p, densityChange=dr)
        self.solver = s

    def capture(self):
        if self.solver is None:
            return
        st = self.solver.getSPH()
        for m, (a, b) in zip(self.members, self.ranges):
            m.state["position"] = st["position"][a:b] - m.offset
            m.state["velocity"] = st["velocity"][a:b]
            m.state["density"] = st["density"][a:b]
            m.state["pressure"] = st["pressure"][a:b]
            m.state["densityChange"] = st["densityChange"][a:b]

    def step(self, n):
        if self.solver is not None and n > 0:
            self.solver.step(n)
            for m in self.members:
                m.steps_done += n

    def num_particles(self):
        return sum(m.scene.fluid.shape[0] for m in self.members)
