"""Drives the reference's own CUDA kernels -- TEST INFRASTRUCTURE ONLY.

oracle/_ref/libdemsph_ref.so is built from the reference sources by
oracle/Makefile.ref.  The classes here replay the reference's host code with
torch-allocated device buffers (torch is only the allocator and stream):

* ``RefSPH`` follows WCSPHSolver (DEMSPH/kernel/WCSPHSolver.h): upload
  (:112-125), spatial grid (:127-135), initializeBoundaryCondition (:29-110),
  neighborSearch (:150-285) and the two half steps (:287-358), including the
  reference's host read of the pair count after each count kernel
  (interaction.h:164-175).
* ``RefDEMPairs`` runs DEMSolver::neighborSearch (DEMSolver.h:698-777) and
  calculateBallContactForceTorque (:599-695) for balls without walls.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libdemsph_ref.so")


class D3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class I3(C.Structure):
    _fields_ = [("x", C.c_int), ("y", C.c_int), ("z", C.c_int)]


_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        p, sz, vp = C.c_void_p, C.c_size_t, C.c_void_p
        L.launchUpdateSpatialGridCellHashStartEnd.argtypes = [p, p, p, p, p, D3, D3, D3, I3, sz, sz, sz, sz, vp]
        L.launchCountSPHInteractions.argtypes = [p, p, p, p, p, p, p, D3, D3, I3, sz, sz, sz, vp]
        L.launchWriteSPHInteractions.argtypes = [p, p, p, p, p, p, p, p, D3, D3, I3, sz, sz, sz, vp]
        L.launchCountSPHDummyInteractions.argtypes = [p, p, p, p, p, p, p, p, p, D3, D3, I3, sz, sz, sz, vp]
        L.launchWriteSPHDummyInteractions.argtypes = [p, p, p, p, p, p, p, p, p, p, D3, D3, I3, sz, sz, sz, vp]
        L.launchCalDummyParticleNormal.argtypes = [p, p, p, p, p, p, p, sz, sz, sz, vp]
        L.launchWCSPH1stHalfIntegration.argtypes = [p] * 22 + [D3, C.c_double, sz, sz, sz, vp]
        L.launchWCSPH2ndHalfIntegration.argtypes = [p] * 23 + [D3, C.c_double, sz, sz, sz, vp]
        L.launchCountBallInteractions.argtypes = [p, p, p, p, p, p, p, p, p, D3, D3, I3, sz, sz, sz, vp]
        L.launchWriteBallInteractions.argtypes = [p] * 20 + [D3, D3, I3, sz, sz, sz, vp]
        L.luanchCalculateBallContactForceTorque.argtypes = [p] * 16 + [C.c_double, sz, sz, sz, vp]
        L.luanchSumBallContactForceTorque.argtypes = [p] * 10 + [sz, sz, sz, vp]
        L.buildHashStartEnd.argtypes = [p, p, p, p, sz, sz, sz, sz, vp]
        L.ref_set_contact_tables.argtypes = [C.c_int, p, C.c_int, p, C.c_int, p, vp]
        L.launchBuildDummyPosition.argtypes = [p, p, D3, D3, D3, I3, sz, sz, sz, vp]
        L.launchUpdateDummySpatialGridCellHashStartEnd.argtypes = [p, p, p, p, p, D3, D3, D3, I3, sz, sz, sz, sz, vp]
        for f in ("launchBuildDummyPosition", "launchUpdateDummySpatialGridCellHashStartEnd",
                  "launchUpdateSpatialGridCellHashStartEnd", "launchCountSPHInteractions",
                  "launchWriteSPHInteractions", "launchCountSPHDummyInteractions", "launchWriteSPHDummyInteractions",
                  "launchCalDummyParticleNormal", "launchWCSPH1stHalfIntegration", "launchWCSPH2ndHalfIntegration",
                  "launchCountBallInteractions", "launchWriteBallInteractions",
                  "luanchCalculateBallContactForceTorque", "luanchSumBallContactForceTorque", "buildHashStartEnd",
                  "ref_set_contact_tables"):
            getattr(L, f).restype = None
        _lib = L
    return _lib


def grid_set(mn, mx, cell):
    """spatialGrid::set (DEMSPH/kernel/boundary.h:70-94)."""
    mn, mx = np.asarray(mn, float), np.asarray(mx, float)
    d = mx - mn
    n = [int(d[k] / cell) if d[k] > cell else 1 for k in range(3)]
    cs = [d[k] / n[k] for k in range(3)]
    return D3(*mn), D3(*mx), D3(*cs), I3(*n), n[0] * n[1] * n[2]


def _launch_dims(n, maxThread=256):
    b = maxThread if maxThread < n else n
    b = max(b, 1)
    return (n + b - 1) // b, b


class _Buf:
    def __init__(self, torch, dev):
        self.t, self.dev = torch, dev

    def f64(self, a, shape=None):
        x = self.t.tensor(np.ascontiguousarray(a, np.float64), device=self.dev)
        return x.reshape(shape) if shape is not None else x

    def zeros(self, shape, dtype):
        return self.t.zeros(shape, dtype=dtype, device=self.dev)


def P(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class RefSPH:
    """WCSPHSolver replayed on the reference kernels."""

    def __init__(self, scene, torch):
        L = lib()
        self.t = torch
        self.dev = torch.device("cuda")
        self.stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        b = _Buf(torch, self.dev)
        nf, nd = scene.fluid.shape[0], scene.dummy.shape[0]
        self.nf, self.nd = nf, nd
        sp, c, rho, nu = scene.spacing, scene.sound_speed, scene.density, scene.viscosity
        f64 = torch.float64
        i32 = torch.int32

        def particles(pos, n):
            d = {}
            d["pos"] = b.f64(pos, (n, 3))
            d["vel"] = b.zeros((n, 3), f64)
            d["acc"] = b.zeros((n, 3), f64)
            d["normal"] = b.zeros((n, 3), f64)
            d["drho"] = b.zeros(n, f64)
            d["rho"] = b.f64(np.full(n, rho))
            d["p"] = b.zeros(n, f64)
            d["rho0"] = b.f64(np.full(n, rho))
            d["h"] = b.f64(np.full(n, 1.3 * sp))
            d["m"] = b.f64(np.full(n, sp ** 3 * rho))
            d["c"] = b.f64(np.full(n, c))
            d["nu"] = b.f64(np.full(n, nu))
            d["hashIndex"] = b.zeros(max(n, 1), i32)
            d["hashValue"] = b.zeros(max(n, 1), i32)
            return d

        self.f = particles(scene.fluid, nf)
        self.d = particles(scene.dummy, nd)
        cell = 2.0 * 1.3 * sp
        self.mn, self.mx, self.cs, self.gs, self.ng = grid_set(scene.minb, scene.maxb, cell)
        self.cellStart = b.zeros(self.ng, i32)
        self.cellEnd = b.zeros(self.ng, i32)
        self.g = D3(*scene.gravity)
        self.dt = scene.dt

        def inter(n, cap):
            return {"count": b.zeros(max(n, 1), i32), "prefix": b.zeros(max(n, 1), i32),
                    "pointed": b.zeros(max(cap, 1), i32), "pointing": b.zeros(max(cap, 1), i32), "cap": cap}

        self.ff = inter(nf, 80 * nf)
        self.fd = inter(nf, 80 * nf)
        self.dd = inter(nd, 80 * nd)
        self.fgrid = _launch_dims(nf)
        self.dgrid = _launch_dims(nd)
        self._init_boundary()

    def _npairs(self, it, n):
        self.t.cuda.synchronize()
        return int(it["prefix"][n - 1].item()) if n > 0 else 0

    def _grow(self, it, need):
        if need > it["cap"]:
            it["pointed"] = self.t.zeros(need, dtype=self.t.int32, device=self.dev)
            it["pointing"] = self.t.zeros(need, dtype=self.t.int32, device=self.dev)
            it["cap"] = need

    def _hash(self, d, n, grid):
        lib().launchUpdateSpatialGridCellHashStartEnd(P(d["pos"]), P(d["hashIndex"]), P(d["hashValue"]),
                                                      P(self.cellStart), P(self.cellEnd), self.mn, self.mx, self.cs,
                                                      self.gs, self.ng, n, grid[0], grid[1], self.stream)

    def _init_boundary(self):
        L = lib()
        d, nd = self.d, self.nd
        if nd == 0:
            return
        self._hash(d, nd, self.dgrid)
        L.launchCountSPHInteractions(P(d["pos"]), P(d["h"]), P(d["hashIndex"]), P(self.dd["count"]),
                                     P(self.dd["prefix"]), P(self.cellStart), P(self.cellEnd), self.mn, self.cs,
                                     self.gs, nd, self.dgrid[0], self.dgrid[1], self.stream)
        self._grow(self.dd, self._npairs(self.dd, nd))
        L.launchWriteSPHInteractions(P(d["pos"]), P(d["h"]), P(d["hashIndex"]), P(self.dd["prefix"]),
                                     P(self.dd["pointed"]), P(self.dd["pointing"]), P(self.cellStart),
                                     P(self.cellEnd), self.mn, self.cs, self.gs, nd, self.dgrid[0], self.dgrid[1],
                                     self.stream)
        L.launchCalDummyParticleNormal(P(d["normal"]), P(d["pos"]), P(d["rho"]), P(d["m"]), P(d["h"]),
                                       P(self.dd["prefix"]), P(self.dd["pointing"]), nd, self.dgrid[0],
                                       self.dgrid[1], self.stream)

    def neighbor_search(self):
        L = lib()
        f, d, nf, nd = self.f, self.d, self.nf, self.nd
        self._hash(f, nf, self.fgrid)
        L.launchCountSPHInteractions(P(f["pos"]), P(f["h"]), P(f["hashIndex"]), P(self.ff["count"]),
                                     P(self.ff["prefix"]), P(self.cellStart), P(self.cellEnd), self.mn, self.cs,
                                     self.gs, nf, self.fgrid[0], self.fgrid[1], self.stream)
        self._grow(self.ff, self._npairs(self.ff, nf))
        L.launchWriteSPHInteractions(P(f["pos"]), P(f["h"]), P(f["hashIndex"]), P(self.ff["prefix"]),
                                     P(self.ff["pointed"]), P(self.ff["pointing"]), P(self.cellStart),
                                     P(self.cellEnd), self.mn, self.cs, self.gs, nf, self.fgrid[0], self.fgrid[1],
                                     self.stream)
        if nd == 0:
            return
        self._hash(d, nd, self.dgrid)
        L.launchCountSPHDummyInteractions(P(f["pos"]), P(f["h"]), P(self.fd["count"]), P(self.fd["prefix"]),
                                          P(d["pos"]), P(d["h"]), P(d["hashIndex"]), P(self.cellStart),
                                          P(self.cellEnd), self.mn, self.cs, self.gs, nf, self.fgrid[0],
                                          self.fgrid[1], self.stream)
        self._grow(self.fd, self._npairs(self.fd, nf))
        L.launchWriteSPHDummyInteractions(P(f["pos"]), P(f["h"]), P(self.fd["prefix"]), P(d["pos"]), P(d["h"]),
                                          P(d["hashIndex"]), P(self.fd["pointed"]), P(self.fd["pointing"]),
                                          P(self.cellStart), P(self.cellEnd), self.mn, self.cs, self.gs, nf,
                                          self.fgrid[0], self.fgrid[1], self.stream)

    def _half(self, second):
        L = lib()
        f, d = self.f, self.d
        common = [P(f["pos"]), P(f["vel"]), P(f["acc"])]
        if second:
            common.append(P(f["drho"]))
        common += [P(f["rho"]), P(f["p"]), P(f["c"]), P(f["m"]), P(f["rho0"]), P(f["h"]), P(f["nu"]),
                   P(self.ff["prefix"]), P(self.fd["prefix"]), P(d["pos"]), P(d["vel"]), P(d["normal"]),
                   P(d["c"]), P(d["m"]), P(d["rho0"]), P(d["h"]), P(d["nu"]), P(self.ff["pointing"]),
                   P(self.fd["pointing"])]
        fn = L.launchWCSPH2ndHalfIntegration if second else L.launchWCSPH1stHalfIntegration
        fn(*common, self.g, self.dt, self.nf, self.fgrid[0], self.fgrid[1], self.stream)

    def step(self, n=1):
        """WCSPHSolver::solve loop body (WCSPHSolver.h:607-621)."""
        for _ in range(n):
            self.neighbor_search()
            self._half(False)
            self._half(True)

    def pairs(self, which):
        it = self.ff if which == 0 else (self.fd if which == 1 else self.dd)
        n = self.nf if which in (0, 1) else self.nd
        k = self._npairs(it, n)
        return it["pointed"][:k].cpu().numpy(), it["pointing"][:k].cpu().numpy()

    def state(self):
        self.t.cuda.synchronize()
        f = self.f
        return {"pos": f["pos"].cpu().numpy(), "vel": f["vel"].cpu().numpy(), "acc": f["acc"].cpu().numpy(),
                "rho": f["rho"].cpu().numpy(), "p": f["p"].cpu().numpy(), "drho": f["drho"].cpu().numpy(),
                "dummy_normal": self.d["normal"].cpu().numpy()}


class RefDEMPairs:
    """DEMSolver::neighborSearch + calculateBallContactForceTorque for balls only
    (no walls, bonds or clumps), from a given ball state."""

    def __init__(self, scene, torch):
        L = lib()
        self.t = torch
        self.dev = torch.device("cuda")
        self.stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        b = _Buf(torch, self.dev)
        n = scene.position.shape[0]
        self.n = n
        f64, i32 = torch.float64, torch.int32
        self.pos = b.f64(scene.position, (n, 3))
        self.vel = b.f64(np.zeros((n, 3)) if scene.velocity is None else scene.velocity, (n, 3))
        w = getattr(scene, "angvel", None)
        self.w = b.f64(np.zeros((n, 3)) if w is None else w, (n, 3))
        self.rad = b.f64(scene.radius)
        m = 4.0 / 3.0 * scene.radius ** 3 * np.pi * scene.density
        self.invm = b.f64(np.where(m > 0, 1.0 / np.where(m > 0, m, 1), 0.0))
        self.mat = torch.tensor(np.asarray(scene.material, np.int32), device=self.dev)
        self.clump = torch.full((n,), -1, dtype=i32, device=self.dev)
        self.force = b.zeros((n, 3), f64)
        self.torque = b.zeros((n, 3), f64)
        self.hashIndex = b.zeros(n, i32)
        self.hashValue = b.zeros(n, i32)
        cell = 2.0 * float(scene.radius.max())
        self.mn, self.mx, self.cs, self.gs, self.ng = grid_set(scene.minb, scene.maxb, cell)
        self.cellStart = b.zeros(self.ng, i32)
        self.cellEnd = b.zeros(self.ng, i32)
        self.count = b.zeros(n, i32)
        self.prefix = b.zeros(n, i32)
        self.iStart = torch.full((n,), -1, dtype=i32, device=self.dev)
        self.iEnd = torch.full((n,), -1, dtype=i32, device=self.dev)
        self.grid = _launch_dims(n)
        rows = lambda rs, k: np.ascontiguousarray(np.array(rs, float).reshape(-1, k)) if rs else np.zeros((1, k))
        h, lr, bd = rows(scene.hertz, 10), rows(scene.linear, 13), rows(scene.bonded, 8)
        L.ref_set_contact_tables(len(scene.hertz), h.ctypes.data_as(C.c_void_p), len(scene.linear),
                                 lr.ctypes.data_as(C.c_void_p), len(scene.bonded), bd.ctypes.data_as(C.c_void_p),
                                 self.stream)
        self.P = 0

    def neighbor_search(self):
        """Fresh lists (no previous list to carry springs from)."""
        L, t, n = lib(), self.t, self.n
        L.launchUpdateSpatialGridCellHashStartEnd(P(self.pos), P(self.hashIndex), P(self.hashValue),
                                                  P(self.cellStart), P(self.cellEnd), self.mn, self.mx, self.cs,
                                                  self.gs, self.ng, n, self.grid[0], self.grid[1], self.stream)
        L.launchCountBallInteractions(P(self.pos), P(self.rad), P(self.invm), P(self.clump), P(self.hashIndex),
                                      P(self.count), P(self.prefix), P(self.cellStart), P(self.cellEnd), self.mn,
                                      self.cs, self.gs, n, self.grid[0], self.grid[1], self.stream)
        t.cuda.synchronize()
        Pn = int(self.prefix[n - 1].item())
        self.P = Pn
        cap = max(Pn, 1)
        f64, i32 = t.float64, t.int32
        z3 = lambda: t.zeros((cap, 3), dtype=f64, device=self.dev)
        self.sl, self.ro, self.to = z3(), z3(), z3()
        self.cF, self.cT, self.cP, self.cN = z3(), z3(), z3(), z3()
        self.ov = t.zeros(cap, dtype=f64, device=self.dev)
        self.pointed = t.zeros(cap, dtype=i32, device=self.dev)
        self.pointing = t.zeros(cap, dtype=i32, device=self.dev)
        oldHash = t.full((cap,), -1, dtype=i32, device=self.dev)
        oldPointed = t.zeros(cap, dtype=i32, device=self.dev)
        L.launchWriteBallInteractions(P(self.pos), P(self.rad), P(self.invm), P(self.clump), P(self.hashIndex),
                                      P(self.prefix), P(self.iStart), P(self.iEnd), P(self.sl), P(self.ro),
                                      P(self.to), P(self.pointed), P(self.pointing), P(self.sl), P(self.ro),
                                      P(self.to), P(oldPointed), P(oldHash), P(self.cellStart), P(self.cellEnd),
                                      self.mn, self.cs, self.gs, n, self.grid[0], self.grid[1], self.stream)
        # buildObjectPointingInteractionStartEnd (DEMSolver.h:59-78)
        self.pHash = t.full((cap,), -1, dtype=i32, device=self.dev)
        pValue = self.pointing.clone()
        pg = _launch_dims(max(Pn, 1))
        if Pn > 0:
            L.buildHashStartEnd(P(self.iStart), P(self.iEnd), P(self.pHash), P(pValue), n, Pn, pg[0], pg[1],
                                self.stream)

    def forces(self, dt):
        """calculateBallContactForceTorque(dt) (DEMSolver.h:599-695) without bonds."""
        L, n = lib(), self.n
        self.force.zero_()
        self.torque.zero_()
        if self.P > 0:
            g = _launch_dims(self.P)
            L.luanchCalculateBallContactForceTorque(P(self.pos), P(self.vel), P(self.w), P(self.rad), P(self.invm),
                                                    P(self.mat), P(self.sl), P(self.ro), P(self.to), P(self.cF),
                                                    P(self.cT), P(self.cP), P(self.cN), P(self.ov), P(self.pointed),
                                                    P(self.pointing), dt, self.P, g[0], g[1], self.stream)
        L.luanchSumBallContactForceTorque(P(self.pos), P(self.force), P(self.torque), P(self.prefix), P(self.iStart),
                                          P(self.iEnd), P(self.cF), P(self.cT), P(self.cP), P(self.pHash), n,
                                          self.grid[0], self.grid[1], self.stream)
        self.t.cuda.synchronize()
        return self.force.cpu().numpy(), self.torque.cpu().numpy()

    def pairs(self):
        self.t.cuda.synchronize()
        return self.pointed[:self.P].cpu().numpy(), self.pointing[:self.P].cpu().numpy()

    def ghost_pass(self, direction, dt):
        """addDummyContactForceTorque(periodic, direction, dt) (DEMSolver.h:
        279-426) from fresh lists, adding into force / torque; returns the
        ghost pairs (pointed, pointing) and their contact forces."""
        L, t, n = lib(), self.t, self.n
        f64, i32 = t.float64, t.int32
        dummy = t.zeros((n, 3), dtype=f64, device=self.dev)
        L.launchBuildDummyPosition(P(dummy), P(self.pos), self.mn, self.mx, self.cs, I3(*direction), n,
                                   self.grid[0], self.grid[1], self.stream)
        L.launchUpdateDummySpatialGridCellHashStartEnd(P(dummy), P(self.hashIndex), P(self.hashValue),
                                                       P(self.cellStart), P(self.cellEnd), self.mn, self.mx, self.cs,
                                                       self.gs, self.ng, n, self.grid[0], self.grid[1], self.stream)
        count = t.zeros(n, dtype=i32, device=self.dev)
        prefix = t.zeros(n, dtype=i32, device=self.dev)
        L.launchCountBallInteractions(P(dummy), P(self.rad), P(self.invm), P(self.clump), P(self.hashIndex),
                                      P(count), P(prefix), P(self.cellStart), P(self.cellEnd), self.mn, self.cs,
                                      self.gs, n, self.grid[0], self.grid[1], self.stream)
        t.cuda.synchronize()
        Pn = int(prefix[n - 1].item())
        cap = max(Pn, 1)
        z3 = lambda: t.zeros((cap, 3), dtype=f64, device=self.dev)
        sl, ro, to, cF, cT, cP, cN = z3(), z3(), z3(), z3(), z3(), z3(), z3()
        ov = t.zeros(cap, dtype=f64, device=self.dev)
        pointed = t.zeros(cap, dtype=i32, device=self.dev)
        pointing = t.zeros(cap, dtype=i32, device=self.dev)
        iStart = t.full((n,), -1, dtype=i32, device=self.dev)
        iEnd = t.full((n,), -1, dtype=i32, device=self.dev)
        oldHash = t.full((cap,), -1, dtype=i32, device=self.dev)
        oldPointed = t.zeros(cap, dtype=i32, device=self.dev)
        L.launchWriteBallInteractions(P(dummy), P(self.rad), P(self.invm), P(self.clump), P(self.hashIndex),
                                      P(prefix), P(iStart), P(iEnd), P(sl), P(ro), P(to), P(pointed), P(pointing),
                                      P(sl), P(ro), P(to), P(oldPointed), P(oldHash), P(self.cellStart),
                                      P(self.cellEnd), self.mn, self.cs, self.gs, n, self.grid[0], self.grid[1],
                                      self.stream)
        pHash = t.full((cap,), -1, dtype=i32, device=self.dev)
        if Pn > 0:
            pValue = pointing.clone()
            pg = _launch_dims(Pn)
            L.buildHashStartEnd(P(iStart), P(iEnd), P(pHash), P(pValue), n, Pn, pg[0], pg[1], self.stream)
            g = _launch_dims(Pn)
            L.luanchCalculateBallContactForceTorque(P(dummy), P(self.vel), P(self.w), P(self.rad), P(self.invm),
                                                    P(self.mat), P(sl), P(ro), P(to), P(cF), P(cT), P(cP), P(cN),
                                                    P(ov), P(pointed), P(pointing), dt, Pn, g[0], g[1], self.stream)
        L.luanchSumBallContactForceTorque(P(dummy), P(self.force), P(self.torque), P(prefix), P(iStart), P(iEnd),
                                          P(cF), P(cT), P(cP), P(pHash), n, self.grid[0], self.grid[1], self.stream)
        t.cuda.synchronize()
        return (pointed[:Pn].cpu().numpy(), pointing[:Pn].cpu().numpy(), cF[:Pn].cpu().numpy())
