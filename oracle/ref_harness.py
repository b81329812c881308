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
* ``RefDEM`` replays DEMSolver for balls, triangle-mesh walls, parallel bonds
  and the buoyancy-drag hook: upload and grids (:155-276), neighborSearch
  with contact-history carry (:698-777, solidInteraction :16-79),
  calculateBallContactForceTorque with bonds (:599-695),
  addTriangleContactForceTorque (:428-597), the external hook
  (externalForceTorque.cu) and the step loops loop_ball / loop_ball_wall
  (:1376-1485).  Clumps are not replayed: the reference's clump force gather
  reads its clump array with a pebble index (ballIntegrationKernel.cu:20),
  past the end of the array.
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
        L.launchCountBallTriangleInteractions.argtypes = [p] * 11 + [D3, D3, I3, sz, sz, sz, vp]
        L.launchWriteBallTriangleInteractions.argtypes = [p] * 22 + [D3, D3, I3, sz, sz, sz, vp]
        L.luanchCalculateBallWallContactForceTorque.argtypes = [p] * 29 + [C.c_double, sz, sz, sz, vp]
        L.luanchCalculateBondedForceTorque.argtypes = [p] * 24 + [C.c_double, sz, sz, sz, vp]
        L.launchBall1stHalfIntegration.argtypes = [p] * 8 + [D3, C.c_double, sz, sz, sz, vp]
        L.launchBall2ndHalfIntegration.argtypes = [p] * 7 + [D3, C.c_double, sz, sz, sz, vp]
        L.launchWallIntegration.argtypes = [p] * 4 + [C.c_double, sz, sz, sz, vp]
        L.launchUpdateWallVertexGlobalPosition.argtypes = [p] * 5 + [sz, sz, sz, vp]
        L.launchUpdateTriangleCircumcenter.argtypes = [p] * 5 + [sz, sz, sz, vp]
        L.launchAddBuoyancyDrag.argtypes = [p] * 5 + [C.c_double, C.c_double, D3, D3, C.c_double, sz, sz, sz, vp]
        L.launchAddConstantForce.argtypes = [p, p, sz, sz, sz, vp]
        L.launchAddGlobalDampingForceTorque.argtypes = [p] * 4 + [C.c_double, sz, sz, sz, vp]
        for f in ("launchCountBallTriangleInteractions", "launchWriteBallTriangleInteractions",
                  "luanchCalculateBallWallContactForceTorque", "luanchCalculateBondedForceTorque",
                  "launchBall1stHalfIntegration", "launchBall2ndHalfIntegration", "launchWallIntegration",
                  "launchUpdateWallVertexGlobalPosition", "launchUpdateTriangleCircumcenter",
                  "launchAddBuoyancyDrag", "launchAddConstantForce", "launchAddGlobalDampingForceTorque"):
            getattr(L, f).restype = None
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


def _cross(a, b):
    """cross (myVec.h), componentwise in the reference's order."""
    return np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1], a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                     a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], axis=1)


def _dot(a, b):
    return a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1] + a[:, 2] * b[:, 2]


def circumcenters(a, b, c):
    """triangleCircumcenter (wallIntegrationKernel.cuh:4-29) for rows of vertices."""
    ab, ac = b - a, c - a
    n = _cross(ab, ac)
    n2 = _dot(n, n)
    t1 = _cross(n, ab) * _dot(ac, ac)[:, None]
    t2 = _cross(ac, n) * _dot(ab, ab)[:, None]
    inv = 1.0 / (2.0 * np.where(n2 < 1e-30, 1.0, n2))
    o = a + (t1 + t2) * inv[:, None]
    return np.where((n2 < 1e-30)[:, None], (a + b + c) / 3.0, o)


class _Solid:
    """solidInteraction (DEMSolver.h:16-79): the pair list with springs and
    contacts, the previous list (oldPair_, oldSpring_), per-pointed-object
    counts / prefix sums and per-pointing-object interaction start / end."""

    def __init__(self, t, dev, n_pointed, n_pointing, cap):
        self.t, self.dev = t, dev
        i32 = t.int32
        self.count = t.zeros(max(n_pointed, 1), dtype=i32, device=dev)
        self.prefix = t.zeros(max(n_pointed, 1), dtype=i32, device=dev)
        self.iStart = t.full((max(n_pointing, 1),), -1, dtype=i32, device=dev)
        self.iEnd = t.full((max(n_pointing, 1),), -1, dtype=i32, device=dev)
        self.n_pointed, self.n_pointing = n_pointed, n_pointing
        self.n = 0
        self._alloc(cap)
        self._alloc_old(cap)

    def _ints(self, cap, fill):
        return self.t.full((max(cap, 1),), fill, dtype=self.t.int32, device=self.dev)

    def _vec(self, cap):
        return self.t.zeros((max(cap, 1), 3), dtype=self.t.float64, device=self.dev)

    def _alloc(self, cap):
        # pair_, spring_, contact_ allocateDevice (interaction.h:40-56, zero fill, ids -1)
        self.pointed, self.pointing = self._ints(cap, -1), self._ints(cap, -1)
        self.hashValue, self.hashIndex, self.cancel = self._ints(cap, -1), self._ints(cap, -1), self._ints(cap, 0)
        self.sl, self.ro, self.to = self._vec(cap), self._vec(cap), self._vec(cap)
        self.cF, self.cT, self.cP, self.cN = self._vec(cap), self._vec(cap), self._vec(cap), self._vec(cap)
        self.ov = self.t.zeros(max(cap, 1), dtype=self.t.float64, device=self.dev)
        self.cap = cap

    def _alloc_old(self, cap):
        self.oPointed, self.oPointing = self._ints(cap, -1), self._ints(cap, -1)
        self.oHashIndex, self.oHashValue, self.oCancel = self._ints(cap, -1), self._ints(cap, -1), self._ints(cap, 0)
        self.oSl, self.oRo, self.oTo = self._vec(cap), self._vec(cap), self._vec(cap)
        self.ocap = cap

    def update_old(self):
        """updateOldPairOldSpring (DEMSolver.h:30-47)."""
        k = self.n
        if k == 0:
            return
        if k > self.ocap:
            self._alloc_old(k)
        for dst, src in ((self.oPointed, self.pointed), (self.oPointing, self.pointing),
                         (self.oHashIndex, self.hashIndex), (self.oHashValue, self.hashValue),
                         (self.oCancel, self.cancel), (self.oSl, self.sl), (self.oRo, self.ro), (self.oTo, self.to)):
            dst[:k].copy_(src[:k])

    def resize(self):
        """resizePair (DEMSolver.h:49-58): the host reads the pair count."""
        self.t.cuda.synchronize()
        self.n = int(self.prefix[self.n_pointed - 1].item()) if self.n_pointed > 0 else 0
        if self.n > self.cap:
            self._alloc(self.n)

    def build_pointing(self, stream, reset=False):
        """buildObjectPointingInteractionStartEnd (DEMSolver.h:60-78).  The
        reference sets interactionStart / End to -1 only when it allocates
        them (interaction.h:73-84), so an object that lost all its pairs
        keeps a range into an older list (quirk Q7); reset=True clears them
        first, as this library's reverse lists are rebuilt from scratch."""
        if reset:
            self.iStart.fill_(-1)
            self.iEnd.fill_(-1)
        if self.n == 0:
            return
        self.hashIndex.fill_(-1)
        self.hashValue.fill_(-1)
        self.hashValue[:self.n].copy_(self.pointing[:self.n])
        g = _launch_dims(self.n)
        lib().buildHashStartEnd(P(self.iStart), P(self.iEnd), P(self.hashIndex), P(self.hashValue), self.n_pointing,
                                self.n, g[0], g[1], stream)


class RefDEM:
    """DEMSolver replayed on the reference's kernels: balls (fixed or free),
    triangle-mesh walls, parallel bonds on the initial contacts, and the
    external hook of the examples (constant force, global damping, buoyancy +
    drag).  No clumps (see the module docstring)."""

    def __init__(self, scene, torch):
        if scene.clumps:
            raise ValueError("RefDEM does not replay clumps")
        L = lib()
        t = self.t = torch
        dev = self.dev = torch.device("cuda")
        self.stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        f64, i32 = t.float64, t.int32
        n = self.n = scene.position.shape[0]
        fixed = np.zeros(n, bool) if scene.fixed is None else np.asarray(scene.fixed, bool)
        r = np.asarray(scene.radius, float)
        rho = np.asarray(scene.density, float)
        # addBall / addFixedBall (DEMSolver.h:1728-1768)
        mass = 4. / 3. * r * r * r * np.pi * rho
        invm = np.where((mass > 0.0) & ~fixed, 1.0 / np.where(mass > 0, mass, 1.0), 0.0)
        vel = np.zeros((n, 3)) if scene.velocity is None else np.asarray(scene.velocity, float)
        w = getattr(scene, "angvel", None)
        w = np.zeros((n, 3)) if w is None else np.asarray(w, float)
        vel = np.where(fixed[:, None], 0.0, vel)
        w = np.where(fixed[:, None], 0.0, w)
        tt = lambda a, shape=None: t.tensor(np.ascontiguousarray(a, np.float64), device=dev).reshape(
            shape if shape is not None else -1)
        self.pos, self.vel, self.w = tt(scene.position, (n, 3)), tt(vel, (n, 3)), tt(w, (n, 3))
        self.force = t.zeros((n, 3), dtype=f64, device=dev)
        self.torque = t.zeros((n, 3), dtype=f64, device=dev)
        self.rad, self.invm = tt(r), tt(invm)
        self.mat = t.tensor(np.asarray(scene.material, np.int32), device=dev)
        self.clump = t.full((n,), -1, dtype=i32, device=dev)
        self.hashIndex = t.zeros(n, dtype=i32, device=dev)
        self.hashValue = t.zeros(n, dtype=i32, device=dev)
        self.grid = _launch_dims(n)
        rows = lambda rs, k: np.ascontiguousarray(np.array(rs, float).reshape(-1, k)) if rs else np.zeros((1, k))
        h, lr, bd = rows(scene.hertz, 10), rows(scene.linear, 13), rows(scene.bonded, 8)
        L.ref_set_contact_tables(len(scene.hertz), h.ctypes.data_as(C.c_void_p), len(scene.linear),
                                 lr.ctypes.data_as(C.c_void_p), len(scene.bonded), bd.ctypes.data_as(C.c_void_p),
                                 self.stream)
        # mesh walls (addMeshWall, DEMSolver.h:1882-1935)
        vl, vw, tri, tw, wpos, wvel, wang, wmat = [], [], [], [], [], [], [], []
        for k, wl in enumerate(scene.walls):
            v0 = len(vl)
            verts = np.asarray(wl["vertices"], float)
            vl += list(verts)
            vw += [k] * len(verts)
            for a, b, c in zip(wl["tri0"], wl["tri1"], wl["tri2"]):
                tri.append((a + v0, b + v0, c + v0))
                tw.append(k)
            wpos.append(np.asarray(wl["position"], float))
            wvel.append(np.asarray(wl.get("velocity", (0, 0, 0)), float))
            wang.append(np.asarray(wl.get("angularVelocity", (0, 0, 0)), float))
            wmat.append(int(wl["material"]))
        self.nw, self.nv, self.nt = len(wpos), len(vl), len(tri)
        cell = 2.0 * float(r.max())
        tcell = cell
        if self.nt:
            vl = np.array(vl)
            tri = np.array(tri, np.int64)
            a, b, c = vl[tri[:, 0]], vl[tri[:, 1]], vl[tri[:, 2]]
            cc = circumcenters(a, b, c)
            for v in (a, b, c):
                tcell = max(tcell, float((2.0 * np.sqrt(_dot(v - cc, v - cc))).max()))
            vg = vl + np.array(wpos)[np.array(vw)]
            ga, gb, gc = vg[tri[:, 0]], vg[tri[:, 1]], vg[tri[:, 2]]
            self.wpos, self.wvel, self.ww = tt(np.array(wpos), (-1, 3)), tt(np.array(wvel), (-1, 3)), tt(
                np.array(wang), (-1, 3))
            self.wq = tt(np.tile([1.0, 0, 0, 0], (self.nw, 1)), (-1, 4))
            self.wmat = t.tensor(np.array(wmat, np.int32), device=dev)
            self.vlocal, self.vglobal = tt(vl, (-1, 3)), tt(vg, (-1, 3))
            self.vwall = t.tensor(np.array(vw, np.int32), device=dev)
            self.i0, self.i1, self.i2 = [t.tensor(tri[:, j].astype(np.int32), device=dev) for j in range(3)]
            self.twall = t.tensor(np.array(tw, np.int32), device=dev)
            self.tcenter = tt(circumcenters(ga, gb, gc), (-1, 3))
            self.thashIndex = t.zeros(self.nt, dtype=i32, device=dev)
            self.thashValue = t.zeros(self.nt, dtype=i32, device=dev)
            self.tg = grid_set(scene.minb, scene.maxb, tcell)
            self.tCellStart = t.zeros(self.tg[4], dtype=i32, device=dev)
            self.tCellEnd = t.zeros(self.tg[4], dtype=i32, device=dev)
            self.bt = _Solid(t, dev, n, self.nt, 0)
        self.mn, self.mx, self.cs, self.gs, self.ng = grid_set(scene.minb, scene.maxb, cell)
        self.cellStart = t.zeros(self.ng, dtype=i32, device=dev)
        self.cellEnd = t.zeros(self.ng, dtype=i32, device=dev)
        self.bb = _Solid(t, dev, n, n, 6 * n)
        self.nb = 0
        self.g = D3(*scene.gravity)
        self.dt = scene.dt
        self.buoyancy = scene.buoyancy
        cf = getattr(scene, "constant_force", None)
        self.fconst = None if cf is None else tt(cf, (n, 3))
        self.damp = 0.0
        self.iStep, self.time = 0, 0.0
        self.bond_initial_contacts = bool(scene.bond_initial_contacts)
        self.correct_q7 = False

    # ------------------------------------------------------------ pieces --
    def initialize(self):
        """The initialisation part of DEMSolver::solve (DEMSolver.h:1994-1998)."""
        self.neighbor_search()
        self.ball_forces(0.0)
        if self.nt:
            self.wall_forces(0.0)
        if self.bond_initial_contacts:
            self.bond_current_pairs()
        # the second initialize() re-uploads the host arrays: forces start at zero
        self.force.zero_()
        self.torque.zero_()

    def neighbor_search(self):
        """DEMSolver::neighborSearch (DEMSolver.h:698-777)."""
        L, n, bb = lib(), self.n, self.bb
        L.launchUpdateSpatialGridCellHashStartEnd(P(self.pos), P(self.hashIndex), P(self.hashValue),
                                                  P(self.cellStart), P(self.cellEnd), self.mn, self.mx, self.cs,
                                                  self.gs, self.ng, n, self.grid[0], self.grid[1], self.stream)
        bb.update_old()
        L.launchCountBallInteractions(P(self.pos), P(self.rad), P(self.invm), P(self.clump), P(self.hashIndex),
                                      P(bb.count), P(bb.prefix), P(self.cellStart), P(self.cellEnd), self.mn,
                                      self.cs, self.gs, n, self.grid[0], self.grid[1], self.stream)
        bb.resize()
        L.launchWriteBallInteractions(P(self.pos), P(self.rad), P(self.invm), P(self.clump), P(self.hashIndex),
                                      P(bb.prefix), P(bb.iStart), P(bb.iEnd), P(bb.sl), P(bb.ro), P(bb.to),
                                      P(bb.pointed), P(bb.pointing), P(bb.oSl), P(bb.oRo), P(bb.oTo),
                                      P(bb.oPointed), P(bb.oHashIndex), P(self.cellStart), P(self.cellEnd), self.mn,
                                      self.cs, self.gs, n, self.grid[0], self.grid[1], self.stream)
        bb.build_pointing(self.stream, self.correct_q7)

    def bond_current_pairs(self):
        """addInitialCondition of the bonded examples (bondedParticleBeam.cpp:
        44-51): bonds on the current contact pairs (bondedInteraction::add,
        DEMSolver.h:93-135), created from the host copy of the positions."""
        a, b = self.pairs(0)
        p = self.pos.cpu().numpy()
        seen, A, B = set(), [], []
        for i0, i1 in zip(a, b):
            if i0 < 0 or i1 < 0 or i0 == i1:
                continue
            x, y = (i0, i1) if i0 < i1 else (i1, i0)
            if (x, y) in seen:
                continue
            seen.add((x, y))
            A.append(x)
            B.append(y)
        A, B = np.array(A, np.int32), np.array(B, np.int32)
        d = p[A] - p[B]
        l2 = d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]
        inv = 1.0 / np.sqrt(np.where(l2 < 1.0e-20, 1.0, l2))
        normal = np.where((l2 < 1.0e-20)[:, None], 0.0, d * inv[:, None])
        t, dev, f64 = self.t, self.dev, self.t.float64
        nb = self.nb = len(A)
        self.bA = t.tensor(A, device=dev)
        self.bB = t.tensor(B, device=dev)
        self.bpoint = t.tensor(0.5 * (p[A] + p[B]), dtype=f64, device=dev)
        self.bnormal = t.tensor(normal, dtype=f64, device=dev)
        z3 = lambda: t.zeros((max(nb, 1), 3), dtype=f64, device=dev)
        z1 = lambda: t.zeros(max(nb, 1), dtype=f64, device=dev)
        self.bFs, self.bTb = z3(), z3()
        self.bFn, self.bTt, self.bsmax, self.btmax = z1(), z1(), z1(), z1()
        self.bok = t.ones(max(nb, 1), dtype=t.int32, device=dev)

    def ball_forces(self, dt):
        """calculateBallContactForceTorque(dt) (DEMSolver.h:599-695)."""
        L, n, bb = lib(), self.n, self.bb
        self.force.zero_()
        self.torque.zero_()
        if bb.n > 0:
            g = _launch_dims(bb.n)
            L.luanchCalculateBallContactForceTorque(P(self.pos), P(self.vel), P(self.w), P(self.rad), P(self.invm),
                                                    P(self.mat), P(bb.sl), P(bb.ro), P(bb.to), P(bb.cF), P(bb.cT),
                                                    P(bb.cP), P(bb.cN), P(bb.ov), P(bb.pointed), P(bb.pointing),
                                                    dt, bb.n, g[0], g[1], self.stream)
        if self.nb > 0:
            g = _launch_dims(self.nb)
            L.luanchCalculateBondedForceTorque(P(self.pos), P(self.vel), P(self.w), P(self.force), P(self.torque),
                                               P(self.rad), P(self.mat), P(bb.prefix), P(bb.cF), P(bb.cT), P(bb.cP),
                                               P(bb.cN), P(bb.pointing), P(self.bpoint), P(self.bnormal),
                                               P(self.bFs), P(self.bTb), P(self.bFn), P(self.bTt), P(self.bsmax),
                                               P(self.btmax), P(self.bok), P(self.bA), P(self.bB), dt, self.nb, g[0],
                                               g[1], self.stream)
        L.luanchSumBallContactForceTorque(P(self.pos), P(self.force), P(self.torque), P(bb.prefix), P(bb.iStart),
                                          P(bb.iEnd), P(bb.cF), P(bb.cT), P(bb.cP), P(bb.hashIndex), n, self.grid[0],
                                          self.grid[1], self.stream)

    def wall_forces(self, dt):
        """addTriangleContactForceTorque(dt) (DEMSolver.h:428-597)."""
        L, n, bt = lib(), self.n, self.bt
        tmn, tmx, tcs, tgs, tng = self.tg
        tgd = _launch_dims(self.nt)
        L.launchUpdateSpatialGridCellHashStartEnd(P(self.tcenter), P(self.thashIndex), P(self.thashValue),
                                                  P(self.tCellStart), P(self.tCellEnd), tmn, tmx, tcs, tgs, tng,
                                                  self.nt, tgd[0], tgd[1], self.stream)
        bt.update_old()
        L.launchCountBallTriangleInteractions(P(self.pos), P(self.rad), P(bt.count), P(bt.prefix), P(self.i0),
                                              P(self.i1), P(self.i2), P(self.thashIndex), P(self.vglobal),
                                              P(self.tCellStart), P(self.tCellEnd), tmn, tcs, tgs, n, self.grid[0],
                                              self.grid[1], self.stream)
        bt.resize()
        L.launchWriteBallTriangleInteractions(P(self.pos), P(self.rad), P(bt.prefix), P(self.i0), P(self.i1),
                                              P(self.i2), P(self.thashIndex), P(bt.iStart), P(bt.iEnd),
                                              P(self.vglobal), P(bt.sl), P(bt.ro), P(bt.to), P(bt.pointed),
                                              P(bt.pointing), P(bt.oSl), P(bt.oRo), P(bt.oTo), P(bt.oPointed),
                                              P(bt.oHashIndex), P(self.tCellStart), P(self.tCellEnd), tmn, tcs, tgs,
                                              n, self.grid[0], self.grid[1], self.stream)
        bt.build_pointing(self.stream, self.correct_q7)
        if bt.n > 0:
            L.luanchCalculateBallWallContactForceTorque(
                P(self.pos), P(self.vel), P(self.w), P(self.force), P(self.torque), P(self.rad), P(self.invm),
                P(self.mat), P(bt.prefix), P(self.wpos), P(self.wvel), P(self.ww), P(self.wmat), P(self.i0),
                P(self.i1), P(self.i2), P(self.twall), P(self.vglobal), P(bt.sl), P(bt.ro), P(bt.to), P(bt.cF),
                P(bt.cT), P(bt.cP), P(bt.cN), P(bt.ov), P(bt.pointed), P(bt.pointing), P(bt.cancel), dt, n,
                self.grid[0], self.grid[1], self.stream)
        wg, vg = _launch_dims(self.nw), _launch_dims(self.nv)
        L.launchWallIntegration(P(self.wpos), P(self.wvel), P(self.ww), P(self.wq), dt, self.nw, wg[0], wg[1],
                                self.stream)
        L.launchUpdateWallVertexGlobalPosition(P(self.vglobal), P(self.vlocal), P(self.vwall), P(self.wpos),
                                               P(self.wq), self.nv, vg[0], vg[1], self.stream)
        L.launchUpdateTriangleCircumcenter(P(self.tcenter), P(self.i0), P(self.i1), P(self.i2), P(self.vglobal),
                                           self.nt, tgd[0], tgd[1], self.stream)

    def external(self, time):
        """addExternalForceTorque of the examples: constant force,
        global damping, buoyancy + drag (externalForceTorque.cu)."""
        L, n = lib(), self.n
        if self.fconst is not None:
            L.launchAddConstantForce(P(self.force), P(self.fconst), n, self.grid[0], self.grid[1], self.stream)
        if self.damp != 0.0:
            L.launchAddGlobalDampingForceTorque(P(self.force), P(self.torque), P(self.vel), P(self.w), self.damp, n,
                                                self.grid[0], self.grid[1], self.stream)
        if self.buoyancy is not None:
            rho, cd, g, u, lvl = self.buoyancy
            L.launchAddBuoyancyDrag(P(self.force), P(self.pos), P(self.vel), P(self.rad), P(self.invm), float(rho),
                                    float(cd), D3(*g), D3(*u), float(lvl), n, self.grid[0], self.grid[1],
                                    self.stream)

    def step(self, num=1):
        """loop_ball / loop_ball_wall (DEMSolver.h:1376-1485)."""
        L, n = lib(), self.n
        hdt = 0.5 * self.dt
        for _ in range(num):
            self.iStep += 1
            self.time += self.dt
            if self.iStep % 5 == 0:
                self.neighbor_search()
            for half in (0, 1):
                self.ball_forces(hdt)
                if self.nt:
                    self.wall_forces(self.dt)
                self.external(self.time - hdt if half == 0 else self.time)
                if half == 0:
                    L.launchBall1stHalfIntegration(P(self.pos), P(self.vel), P(self.w), P(self.force),
                                                   P(self.torque), P(self.rad), P(self.invm), P(self.clump), self.g,
                                                   hdt, n, self.grid[0], self.grid[1], self.stream)
                else:
                    L.launchBall2ndHalfIntegration(P(self.vel), P(self.w), P(self.force), P(self.torque),
                                                   P(self.rad), P(self.invm), P(self.clump), self.g, hdt, n,
                                                   self.grid[0], self.grid[1], self.stream)

    # ------------------------------------------------------------ state --
    def set_balls(self, pos=None, vel=None, w=None):
        for dst, src in ((self.pos, pos), (self.vel, vel), (self.w, w)):
            if src is not None:
                dst.copy_(self.t.tensor(np.asarray(src, float), dtype=self.t.float64, device=self.dev))

    def balls(self):
        self.t.cuda.synchronize()
        return {"pos": self.pos.cpu().numpy(), "vel": self.vel.cpu().numpy(), "angvel": self.w.cpu().numpy(),
                "force": self.force.cpu().numpy(), "torque": self.torque.cpu().numpy()}

    def pairs(self, which=0):
        """(pointed, pointing) of the ball-ball (0) or ball-triangle (1) list."""
        s = self.bb if which == 0 else self.bt
        self.t.cuda.synchronize()
        return s.pointed[:s.n].cpu().numpy(), s.pointing[:s.n].cpu().numpy()

    def springs(self, which=0):
        s = self.bb if which == 0 else self.bt
        self.t.cuda.synchronize()
        return {"a": s.pointed[:s.n].cpu().numpy(), "b": s.pointing[:s.n].cpu().numpy(),
                "sliding": s.sl[:s.n].cpu().numpy(), "rolling": s.ro[:s.n].cpu().numpy(),
                "torsion": s.to[:s.n].cpu().numpy()}

    def bonds(self):
        self.t.cuda.synchronize()
        k = self.nb
        g = lambda x: x[:k].cpu().numpy()
        return {"a": g(self.bA), "b": g(self.bB), "ok": g(self.bok), "normal_force": g(self.bFn),
                "torsion_torque": g(self.bTt), "shear_force": g(self.bFs), "bending_torque": g(self.bTb),
                "normal": g(self.bnormal), "point": g(self.bpoint)}
