"""Batched form: many independent scenes stepped as one device scene.

Each member scene is translated into its own tile of the x-y plane; tiles are
separated by empty cells, so no pair crosses between members and every
member's grid neighbourhood is its own.  The physics is translation
invariant and the cell (>= 2 r_max, >= 2 h_max) still contains every
interacting pair, so a member evolves as it does alone, up to rounding of the
translated coordinates, while all members share one set of kernel launches
per step (one cell sort, one pair pass, one reduction, ...).

Membership changes (admission, retirement) replace the device scene at a
step boundary in two parts.  `prepare(members)` builds and initialises the
next device scene from the members' initial scenes (or host states), on the
batch's other stream, and can run while the current scene is stepping.
`commit(prepared)` then copies the continuing members' state from the
current device scene into the new one with a device kernel (no host round
trip): positions (re-translated), velocities and angular velocities, their
pair rows and ball-triangle rows with the springs (DEM), and density /
pressure / density change (SPH).  DEM members change only at steps that are
multiples of 5, the reference's re-sort cadence (DEMSolver.h:1384), and their
pair rows are copied as they are, so each member uses exactly the pair list it
would use alone.

Members keep the reference's domain-edge behaviour only while their particles
stay inside their own domain box: a particle that leaves it is clamped into
the edge cells of the batch domain rather than of its own.
"""
from __future__ import annotations

import math
import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import scenes as S


@dataclass
class Member:
    key: int
    scene: object
    offset: np.ndarray = None
    steps_done: int = 0
    # host copy of the state (member-local coordinates / indices), filled by
    # capture(); a member with a host state and no device home starts from it
    state: dict = field(default_factory=dict)
    home: object = None        # the device scene holding the member's live state
    record: object = None      # the scene's device-resident member record (assembly source)
    range: tuple = None        # its particle index range there
    tri_range: tuple = None    # its triangle index range there (DEM)
    clump_range: tuple = None  # its clump index range there (DEM)
    bond_range: tuple = None   # its bond index range there (DEM)
    # its bonds (member-local ball indices, the order the device scene holds
    # them in), fixed at its first admission (DEM)
    bonds: tuple = None


@dataclass
class Prepared:
    """A device scene built for a member list, not yet holding their state."""
    solver: object
    members: list
    ranges: list
    tri_ranges: list
    offsets: list
    stream: int
    clump_ranges: list = None  # DEM: each member's clump index range
    bond_ranges: list = None   # DEM: each member's bond index range


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


class _Reaper:
    """Destroys replaced device scenes on a background thread: tearing a
    scene down synchronises its stream and frees its buffers, which need not
    hold up the next chunk."""

    def __init__(self):
        self.q = queue.Queue()
        t = threading.Thread(target=self._run, daemon=True)
        t.start()

    def _run(self):
        while True:
            obj = self.q.get()
            del obj

    def drop(self, obj):
        if obj is not None:
            self.q.put(obj)


_reaper = None


def _drop(obj):
    global _reaper
    if _reaper is None:
        _reaper = _Reaper()
    _reaper.drop(obj)


class _Batch:
    """Member bookkeeping shared by the DEM and WCSPH batches."""

    def __init__(self, precision="mixed", stream=None, streams=None, tuning=None):
        self.precision = precision
        # an autotune.Tuning of this kind: cell size, capacities, list shape
        # and skin of every batch scene
        self.tuning = tuning
        # two streams: the next scene is prepared on the one the current scene
        # does not use
        self.streams = list(streams) if streams is not None else [stream, stream]
        self.cur_stream = 0
        self.members: list[Member] = []
        self.solver = None
        self.ranges = []
        self.tri_ranges = []
        # seconds spent preparing device scenes (build + initialise) and in
        # the state carry, and how many scenes were committed
        self.timing = {"initialize_s": 0.0, "carry_s": 0.0, "rebuilds": 0}

    def _carried(self, prep):
        old = self.solver
        return [(m, k) for k, m in enumerate(prep.members) if old is not None and m.home is old]

    def rebuild(self):
        """prepare + commit of the current member list."""
        if not self.members:
            self.solver = None
            return
        self.commit(self.prepare(self.members))

    def step(self, n):
        """n steps of every member; returns when the device has done them."""
        if self.solver is not None and n > 0:
            self.solver.step(n)
            if hasattr(self.solver, "synchronize"):
                self.solver.synchronize()
            for m in self.members:
                m.steps_done += n

    def clear(self):
        self.solver = None
        self.members = []


def _num_balls(scene):
    """Balls of a DEM member, its clumps' pebbles included (they follow its
    balls, clump by clump)."""
    return scene.position.shape[0] + sum(len(c["radius"]) for c in scene.clumps)


def _initial_positions(scene):
    """Initial positions of a DEM member's balls and pebbles, in device order."""
    parts = [scene.position] + [np.asarray(c["point"], float).reshape(-1, 3) for c in scene.clumps]
    return np.concatenate(parts, axis=0)


class DEMBatch(_Batch):
    """DEM members of one time step and gravity stepped together.  Members
    may hold clumps (their pebbles follow the member's balls), bonds on their
    initial contacts (the addInitialCondition hook of the bonded scenes: the
    member's contacts in the batch's first pair list after its admission)
    and a constant force per ball (no ramp)."""

    @staticmethod
    def cell_of(scene):
        return 2.0 * float(np.max(scene.radius))

    @staticmethod
    def _materials(members):
        """Material ids of the batch: members with the same parameter rows
        share a block of ids, member ids shifted by the block's offset.
        Returns per-member offsets and the shifted rows."""
        sig = {}
        offs = []
        rows_h, rows_l, rows_b = [], [], []
        base = 0
        for m in members:
            sc = m.scene
            key = (tuple(map(tuple, sc.hertz)), tuple(map(tuple, sc.linear)), tuple(map(tuple, sc.bonded)))
            if key not in sig:
                top = max([int(np.max(sc.material))] + [int(w["material"]) for w in sc.walls] +
                          [int(r[i]) for r in sc.hertz + sc.linear + sc.bonded for i in (0, 1)])
                sig[key] = base
                for r in sc.hertz:
                    rows_h.append((base + int(r[0]), base + int(r[1])) + tuple(r[2:]))
                for r in sc.linear:
                    rows_l.append((base + int(r[0]), base + int(r[1])) + tuple(r[2:]))
                for r in sc.bonded:
                    rows_b.append((base + int(r[0]), base + int(r[1])) + tuple(r[2:]))
                base += top + 1
            offs.append(sig[key])
        return offs, rows_h, rows_l, rows_b

    def prepare(self, members):
        """Builds and initialises the device scene for `members`.  Members
        without a host state are assembled on the device from their member
        records (uploaded once, on first use); a member with a host state
        (and no device home) starts from it."""
        from .scenes import DEMScene
        from .solvers import DEMMember, DEMSolver

        tic = time.perf_counter()
        for m in members:
            sc = m.scene
            if sc.periodic is not None or sc.buoyancy is not None:
                raise ValueError("batched DEM members have no periodic boundaries or buoyancy plane")
            if (sc.clumps or sc.bond_initial_contacts) and m.home is None and "position" in m.state:
                raise ValueError("a member with clumps or bonds re-enters a batch only from its device scene")
        cell = max(self.cell_of(m.scene) for m in members)
        boxes = [(np.asarray(m.scene.minb), np.asarray(m.scene.maxb)) for m in members]
        offs = tile_offsets(boxes, gap=2.0 * cell)
        moffs, rows_h, rows_l, rows_b = self._materials(members)
        lo = np.full(3, np.inf)
        hi = np.full(3, -np.inf)
        ranges, tri_ranges, clump_ranges = [], [], []
        start = 0
        tstart = 0
        cstart = 0
        walls = []
        for m, off, mo in zip(members, offs, moffs):
            sc = m.scene
            n = _num_balls(sc)
            clump_ranges.append((cstart, cstart + len(sc.clumps)))
            cstart += len(sc.clumps)
            for wl in sc.walls:
                d = dict(wl)
                d["position"] = np.asarray(wl["position"], float) + off
                d["material"] = mo + int(wl["material"])
                walls.append(d)
            nt = sum(len(wl["tri0"]) for wl in sc.walls)
            ranges.append((start, start + n))
            tri_ranges.append((tstart, tstart + nt))
            start += n
            tstart += nt
            lo = np.minimum(lo, np.asarray(sc.minb) + off)
            hi = np.maximum(hi, np.asarray(sc.maxb) + off)
        first = members[0].scene
        si = 1 - self.cur_stream
        hosted = [m.home is None and "position" in m.state for m in members]
        if not any(hosted):
            new = DEMSolver(self.streams[si])
            if self.tuning is not None:
                self.tuning.configure(new)
            for r in rows_h:
                new.setHertzianPair(*r)
            for r in rows_l:
                new.setLinearPair(*r)
            for r in rows_b:
                new.setBondedPair(*r)
            recs = []
            for m in members:
                if m.record is None:
                    sc = m.scene
                    rec = DEMMember(self.streams[si])
                    fixed = np.zeros(sc.position.shape[0], bool) if sc.fixed is None else sc.fixed
                    w0 = getattr(sc, "angvel", None)
                    # balls in scene order: runs of moving / fixed balls
                    idx = np.flatnonzero(np.diff(np.r_[-1, fixed.astype(int)]) != 0)
                    bounds = list(idx) + [len(fixed)]
                    for a, b in zip(bounds[:-1], bounds[1:]):
                        sl = slice(a, b)
                        rec.addBalls(sc.position[sl], None if sc.velocity is None else sc.velocity[sl],
                                     None if w0 is None else w0[sl], sc.radius[sl], sc.density[sl],
                                     sc.material[sl], fixed=bool(fixed[a]))
                    for c in sc.clumps:
                        rec.addClump(c["point"], c["radius"], c["centroid"], c["velocity"], c["angularVelocity"],
                                     c["mass"], c["inertia"], c["material"])
                    m.record = rec.seal()
                recs.append(m.record)
            new.assembleBalls(recs, offs, moffs)
            for k, wl in enumerate(walls):
                new.addMeshWall(wl["vertices"], wl["tri0"], wl["tri1"], wl["tri2"], wl["position"],
                                materialID=wl["material"])
                if "velocity" in wl:
                    new.setMeshWallMotion(k, wl["velocity"], wl.get("angularVelocity", (0, 0, 0)))
            new.initialize(tuple(lo), tuple(hi), first.gravity, first.dt, self.precision)
            bond_ranges = self._bonds(new, members, ranges, offs)
            self._constant_force(new, members, ranges)
        else:
            if any(m.scene.clumps for m in members):
                raise ValueError("a batch with members entering from a host state holds no clumps")
            pos, vel, w, rad, den, mat, fixed = [], [], [], [], [], [], []
            for m, off, mo, h in zip(members, offs, moffs, hosted):
                sc = m.scene
                st = m.state if h else {}
                n = sc.position.shape[0]
                pos.append((st["position"] if "position" in st else sc.position) + off)
                v0 = sc.velocity if sc.velocity is not None else np.zeros((n, 3))
                w0 = getattr(sc, "angvel", None)
                w0 = w0 if w0 is not None else np.zeros((n, 3))
                vel.append(st.get("velocity", v0))
                w.append(st.get("angularVelocity", w0))
                rad.append(sc.radius)
                den.append(sc.density)
                mat.append(np.asarray(sc.material, np.int32) + mo)
                fixed.append(np.zeros(n, bool) if sc.fixed is None else sc.fixed)
            big = DEMScene(name="batch", position=np.concatenate(pos), radius=np.concatenate(rad),
                           density=np.concatenate(den), material=np.concatenate(mat),
                           velocity=np.concatenate(vel), fixed=np.concatenate(fixed), hertz=rows_h, linear=rows_l,
                           bonded=rows_b, walls=walls, minb=tuple(lo), maxb=tuple(hi), gravity=first.gravity,
                           dt=first.dt)
            big.angvel = np.concatenate(w)
            new = S.build_dem(big, self.precision, self.streams[si],
                              configure=None if self.tuning is None else self.tuning.configure)
            # springs of members entering from a host state, renumbered
            A, B, SL, RO, TO = [], [], [], [], []
            WA, WT, WS, WR, WTo = [], [], [], [], []
            for m, h, (b0, _), (t0, _) in zip(members, hosted, ranges, tri_ranges):
                if not h:
                    continue
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
                new.importSprings(np.concatenate(A), np.concatenate(B), np.concatenate(SL), np.concatenate(RO),
                                  np.concatenate(TO))
            if WA:
                new.importWallSprings(np.concatenate(WA), np.concatenate(WT), np.concatenate(WS),
                                      np.concatenate(WR), np.concatenate(WTo))
            bond_ranges = self._bonds(new, members, ranges, offs)
            self._constant_force(new, members, ranges)
        self.timing["initialize_s"] += time.perf_counter() - tic
        return Prepared(new, list(members), ranges, tri_ranges, offs, si, clump_ranges, bond_ranges)

    @staticmethod
    def _bonds(new, members, ranges, offs):
        """Bonds of the members with bond_initial_contacts, added to the
        initialised scene `new` member by member (each member's bonds one
        block, in the order it keeps them).  A member's bonds are fixed at its
        first admission: its contacts between balls (not pebbles) in `new`'s
        pair list.  Returns each member's bond index range."""
        out = [(0, 0)] * len(members)
        if not any(m.scene.bond_initial_contacts for m in members):
            return out
        pairs = None
        A, B = [], []
        for k, (m, (b0, b1)) in enumerate(zip(members, ranges)):
            if not m.scene.bond_initial_contacts:
                continue
            if m.bonds is None:
                if pairs is None:
                    p = new.getPairs(0)
                    pairs = (p["objectPointed"], p["objectPointing"])
                nb = m.scene.position.shape[0]
                a, b = pairs
                sel = (a >= b0) & (a < b0 + nb) & (b >= b0) & (b < b0 + nb)
                la, lb = a[sel] - b0, b[sel] - b0
                lo_, hi_ = np.minimum(la, lb), np.maximum(la, lb)
                # the library keeps the first of repeated pairs, (min, max) ordered
                _, first = np.unique(lo_.astype(np.int64) * (b1 - b0) + hi_, return_index=True)
                keep = np.sort(first)
                m.bonds = (lo_[keep].astype(np.int32), hi_[keep].astype(np.int32))
            A.append(m.bonds[0] + b0)
            B.append(m.bonds[1] + b0)
        if not A:
            return out
        pos = np.zeros((ranges[-1][1], 3))
        for m, (b0, b1), off in zip(members, ranges, offs):
            pos[b0:b1] = _initial_positions(m.scene) + off
        new.addBondedInteraction(np.concatenate(A), np.concatenate(B), pos)
        start = 0
        for k, m in enumerate(members):
            nb = len(m.bonds[0]) if m.scene.bond_initial_contacts else 0
            out[k] = (start, start + nb)
            start += nb
        return out

    @staticmethod
    def _constant_force(new, members, ranges):
        if not any(getattr(m.scene, "constant_force", None) is not None for m in members):
            return
        f = np.zeros((ranges[-1][1], 3))
        for m, (b0, b1) in zip(members, ranges):
            cf = getattr(m.scene, "constant_force", None)
            if cf is not None:
                cf = np.asarray(cf, float).reshape(-1, 3)
                f[b0:b0 + cf.shape[0]] = cf
        new.setConstantForce(f)

    def commit(self, prep):
        """Carries the continuing members' state from the current device
        scene into the prepared one and makes it current."""
        tic = time.perf_counter()
        old = self.solver
        carried = self._carried(prep)
        if carried:
            ss = [m.range[0] for m, k in carried]
            ds = [prep.ranges[k][0] for m, k in carried]
            nn = [m.range[1] - m.range[0] for m, k in carried]
            td = [prep.tri_ranges[k][0] - m.tri_range[0] for m, k in carried]
            sh = [prep.offsets[k] - m.offset for m, k in carried]
            prep.solver.copyMembers(old, ss, ds, nn, td, sh)
            bodies = [(m, k) for m, k in carried if m.clump_range[1] > m.clump_range[0] or
                      m.bond_range[1] > m.bond_range[0]]
            if bodies:
                prep.solver.copyMemberBodies(
                    old, [m.clump_range[0] for m, k in bodies], [prep.clump_ranges[k][0] for m, k in bodies],
                    [m.clump_range[1] - m.clump_range[0] for m, k in bodies],
                    [m.bond_range[0] for m, k in bodies], [prep.bond_ranges[k][0] for m, k in bodies],
                    [m.bond_range[1] - m.bond_range[0] for m, k in bodies],
                    [prep.offsets[k] - m.offset for m, k in bodies])
        for m, r, t, off, cr, br in zip(prep.members, prep.ranges, prep.tri_ranges, prep.offsets,
                                        prep.clump_ranges, prep.bond_ranges):
            m.home, m.range, m.tri_range, m.offset = prep.solver, r, t, off
            m.clump_range, m.bond_range = cr, br
        self.members = prep.members
        self.ranges, self.tri_ranges = prep.ranges, prep.tri_ranges
        self.solver = prep.solver
        self.cur_stream = prep.stream
        _drop(old)
        del old
        self.timing["carry_s"] += time.perf_counter() - tic
        self.timing["rebuilds"] += 1

    def capture(self, keys=None):
        """Copies the state of the members (or of those in `keys`) out of the
        device scene into their host state."""
        if self.solver is None:
            return
        b = self.solver.getBall()
        pp = self.solver.getPairs(0)
        wp = self.solver.getPairs(1)
        cl = bo = None
        for m, (b0, b1), (t0, t1) in zip(self.members, self.ranges, self.tri_ranges):
            if keys is not None and m.key not in keys:
                continue
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
            c0, c1 = m.clump_range
            if c1 > c0:
                if cl is None:
                    cl = self.solver.getClump()
                st["clumps"] = {"position": cl["position"][c0:c1] - m.offset, "velocity": cl["velocity"][c0:c1],
                                "angularVelocity": cl["angularVelocity"][c0:c1],
                                "orientation": cl["orientation"][c0:c1]}
            k0, k1 = m.bond_range
            if k1 > k0:
                if bo is None:
                    bo = self.solver.getBondedInteraction()
                st["bonds"] = {k: (v[k0:k1] - (b0 if k.startswith("object") else 0)) if v.ndim == 1
                               else (v[k0:k1] - m.offset if k == "point" else v[k0:k1]) for k, v in bo.items()}

    def num_particles(self):
        return sum(m.scene.num_moving for m in self.members)


class SPHBatch(_Batch):
    """WCSPH members of one time step and gravity stepped together."""

    def prepare(self, members):
        """Builds and initialises the device scene for `members` (see
        DEMBatch.prepare).  Members without a host state are assembled on the
        device from their member records (uploaded once, on first use)."""
        from .solvers import SPHMember, WCSPHSolver

        tic = time.perf_counter()
        cell = max(2.0 * 1.3 * m.scene.spacing for m in members)
        boxes = [(np.asarray(m.scene.minb), np.asarray(m.scene.maxb)) for m in members]
        offs = tile_offsets(boxes, gap=2.0 * cell)
        si = 1 - self.cur_stream
        s = WCSPHSolver(self.streams[si])
        if self.tuning is not None:
            self.tuning.configure(s)
        lo = np.full(3, np.inf)
        hi = np.full(3, -np.inf)
        ranges = []
        start = 0
        for m, off in zip(members, offs):
            sc = m.scene
            n = sc.fluid.shape[0]
            ranges.append((start, start + n))
            start += n
            lo = np.minimum(lo, np.asarray(sc.minb) + off)
            hi = np.maximum(hi, np.asarray(sc.maxb) + off)
        first = members[0].scene
        hosted = [m.home is None and "position" in m.state for m in members]
        if not any(hosted):
            recs = []
            for m in members:
                if m.record is None:
                    sc = m.scene
                    r = SPHMember(self.streams[si])
                    r.addSPHs(sc.fluid, None, sc.sound_speed, sc.spacing, sc.density, sc.viscosity)
                    r.addDummies(sc.dummy, None, sc.sound_speed, sc.spacing, sc.density, sc.viscosity)
                    m.record = r.seal()
                recs.append(m.record)
            s.assemble(recs, offs, tuple(lo), tuple(hi), first.gravity, first.dt, self.precision)
        else:
            for m, h, off in zip(members, hosted, offs):
                sc = m.scene
                st = m.state if h else {}
                s.addSPHs(st.get("position", sc.fluid) + off, st.get("velocity"), sc.sound_speed, sc.spacing,
                          sc.density, sc.viscosity)
            for m, off in zip(members, offs):
                sc = m.scene
                s.addDummies(sc.dummy + off, None, sc.sound_speed, sc.spacing, sc.density, sc.viscosity)
            s.initialize(tuple(lo), tuple(hi), first.gravity, first.dt, self.precision)
            if any(h and "density" in m.state for m, h in zip(members, hosted)):
                rho = np.empty(start)
                p = np.empty(start)
                dr = np.empty(start)
                for m, h, (a, b) in zip(members, hosted, ranges):
                    st = m.state if h else {}
                    rho[a:b] = st.get("density", np.full(b - a, m.scene.density))
                    p[a:b] = st.get("pressure", np.zeros(b - a))
                    dr[a:b] = st.get("densityChange", np.zeros(b - a))
                s.setSPH(density=rho, pressure=p, densityChange=dr)
        if self.tuning is not None:
            self.tuning.finish(s)
        self.timing["initialize_s"] += time.perf_counter() - tic
        return Prepared(s, list(members), ranges, [None] * len(members), offs, si)

    def commit(self, prep):
        """Carries the continuing members' fluid state into the prepared
        scene and makes it current."""
        tic = time.perf_counter()
        old = self.solver
        carried = self._carried(prep)
        if carried:
            ss = [m.range[0] for m, k in carried]
            ds = [prep.ranges[k][0] for m, k in carried]
            nn = [m.range[1] - m.range[0] for m, k in carried]
            sh = [prep.offsets[k] - m.offset for m, k in carried]
            prep.solver.copyMembers(old, ss, ds, nn, sh)
        for m, r, off in zip(prep.members, prep.ranges, prep.offsets):
            m.home, m.range, m.offset = prep.solver, r, off
        self.members = prep.members
        self.ranges = prep.ranges
        self.solver = prep.solver
        self.cur_stream = prep.stream
        _drop(old)
        del old
        self.timing["carry_s"] += time.perf_counter() - tic
        self.timing["rebuilds"] += 1

    def capture(self, keys=None):
        if self.solver is None:
            return
        st = self.solver.getSPH()
        for m, (a, b) in zip(self.members, self.ranges):
            if keys is not None and m.key not in keys:
                continue
            m.state["position"] = st["position"][a:b] - m.offset
            m.state["velocity"] = st["velocity"][a:b]
            m.state["density"] = st["density"][a:b]
            m.state["pressure"] = st["pressure"][a:b]
            m.state["densityChange"] = st["densityChange"][a:b]

    def num_particles(self):
        return sum(m.scene.fluid.shape[0] for m in self.members)
