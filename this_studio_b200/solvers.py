"""Python mirror of the reference's solver classes over the C ABI.

``DEMSolver`` follows DEMSPH/kernel/DEMSolver.h (scene setup :1633-1959,
solve :1961-2049, step pieces :278-906, getters :1541-1631) and
``WCSPHSolver`` follows DEMSPH/kernel/WCSPHSolver.h (:522-624), with the same
method names and argument meaning.  ``solve`` runs the reference's step loop
without the VTU output; ``initialize`` + ``step`` split it for callers that
step incrementally.  Bulk adders (``addBalls`` ...) take arrays.

Errors: every native failure raises ``DemsphError`` carrying the status code.
The reference instead returns silently or exits (DEMSolver.h:1974-2004).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import call

_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int)


def _f64(a, shape=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return a.reshape(shape) if shape is not None else a


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def _dp(a):
    return None if a is None else a.ctypes.data_as(_d)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_i)


def _v3(x):
    return _f64(x, (3,))


def _stream_ptr(stream):
    if stream is None or stream == 0:
        return None
    return C.c_void_p(int(getattr(stream, "cuda_stream", stream)))


def num_steps(timeStep, maximumTime):
    """Step count of solve(): size_t(maximumTime / timeStep) + 1 iterations of
    ``while (iStep <= numStep)`` (DEMSolver.h:1988,1380), i.e. numStep + 1."""
    return int(maximumTime / timeStep) + 1 + 1


def _run_frames(solver, total, numFrame, write):
    """The reference's frame cadence (DEMSolver.h:1984-2046, WCSPHSolver.h:
    587-621): frame 0 after initialisation; numStep = total - 1 and
    frameInterval = numStep / numFrame (numStep when numFrame is 0, at least
    1); after step iStep (1-based), frame += 1 whenever iStep % frameInterval
    == 0."""
    num_step = total - 1
    interval = num_step // numFrame if numFrame > 0 else num_step
    interval = max(1, interval)
    write(0)
    done = 0
    frame = 0
    while done < total:
        nxt = min(total, (done // interval + 1) * interval)
        solver.step(nxt - done)
        done = nxt
        if done % interval == 0:
            frame += 1
            write(frame)


class DEMMember:
    """One scene's balls held on the device, from which batch scenes are
    assembled (DEMSolver.assembleBalls)."""

    def __init__(self, stream=None):
        self._h = C.c_void_p()
        call("demsph_dem_member_create", C.byref(self._h), _stream_ptr(stream))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().demsph_dem_member_destroy(h)
            except Exception:
                pass
            self._h = None

    def addBalls(self, position, velocity, angularVelocity, radius, density, materialID, fixed=False):
        p = _f64(position, (-1, 3))
        n = p.shape[0]
        v = None if velocity is None else _f64(velocity, (n, 3))
        w = None if angularVelocity is None else _f64(angularVelocity, (n, 3))
        r = _f64(np.broadcast_to(radius, (n,)))
        d = None if density is None else _f64(np.broadcast_to(density, (n,)))
        m = _i32(np.broadcast_to(materialID, (n,)))
        call("demsph_dem_member_add_balls", self._h, n, _dp(p), _dp(v), _dp(w), _dp(r), _dp(d), _ip(m), int(fixed))

    def addClump(self, point, radius, centroidPosition, velocity, angularVelocity, mass, inertiaTensor, materialID):
        """DEMSolver.addClump into the member: pebbles follow the balls added so far."""
        p = _f64(point, (-1, 3))
        call("demsph_dem_member_add_clump", self._h, p.shape[0], _dp(p), _dp(_f64(radius)),
             _dp(_v3(centroidPosition)), _dp(_v3(velocity)), _dp(_v3(angularVelocity)), float(mass),
             _dp(_f64(inertiaTensor, (6,))), int(materialID))

    def seal(self):
        call("demsph_dem_member_seal", self._h)
        return self

    def num(self):
        n = C.c_long()
        call("demsph_dem_member_count", self._h, C.byref(n))
        return n.value

    def numClumps(self):
        n = C.c_long()
        call("demsph_dem_member_num_clumps", self._h, C.byref(n))
        return n.value


class DEMSolver:
    """Spheres, clumps, triangle-mesh walls, linear / Hertz-Mindlin / bonded contact."""

    def __init__(self, stream=None):
        self._h = C.c_void_p()
        call("demsph_dem_create", C.byref(self._h), _stream_ptr(stream))
        self._nvert = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().demsph_dem_destroy(h)
            except Exception:
                pass
            self._h = None

    # ---------------------------------------------------------- materials --
    def setHertzianPair(self, materialIndexA, materialIndexB, effectiveYoungsModulus, effectiveShearModulus,
                        restitutionCoefficient, rollingStiffnessToShearStiffnessRatio=0.0,
                        torsionStiffnessToShearStiffnessRatio=0.0, slidingFrictionCoefficient=0.0,
                        rollingFrictionCoefficient=0.0, torsionFrictionCoefficient=0.0):
        call("demsph_dem_set_hertzian_pair", self._h, materialIndexA, materialIndexB, effectiveYoungsModulus,
             effectiveShearModulus, restitutionCoefficient, rollingStiffnessToShearStiffnessRatio,
             torsionStiffnessToShearStiffnessRatio, slidingFrictionCoefficient, rollingFrictionCoefficient,
             torsionFrictionCoefficient)

    def setLinearPair(self, materialIndexA, materialIndexB, normalStiffness, slidingStiffness, rollingStiffness,
                      torsionStiffness, normalDissipation, slidingDissipation, rollingDissipation, torsionDissipation,
                      slidingFrictionCoefficient, rollingFrictionCoefficient, torsionFrictionCoefficient):
        call("demsph_dem_set_linear_pair", self._h, materialIndexA, materialIndexB, normalStiffness,
             slidingStiffness, rollingStiffness, torsionStiffness, normalDissipation, slidingDissipation,
             rollingDissipation, torsionDissipation, slidingFrictionCoefficient, rollingFrictionCoefficient,
             torsionFrictionCoefficient)

    def setBondedPair(self, materialIndexA, materialIndexB, bondRadiusMultiplier, bondYoungsModulus,
                      normalToShearStiffnessRatio, tensileStrength, cohesion, frictionCoefficient):
        call("demsph_dem_set_bonded_pair", self._h, materialIndexA, materialIndexB, bondRadiusMultiplier,
             bondYoungsModulus, normalToShearStiffnessRatio, tensileStrength, cohesion, frictionCoefficient)

    # ------------------------------------------------------------- bodies --
    def addBalls(self, position, velocity, angularVelocity, radius, density, materialID, clumpID=None):
        p = _f64(position, (-1, 3))
        n = p.shape[0]
        v = _f64(np.zeros((n, 3)) if velocity is None else velocity, (n, 3))
        w = _f64(np.zeros((n, 3)) if angularVelocity is None else angularVelocity, (n, 3))
        r = _f64(np.broadcast_to(radius, (n,)))
        d = _f64(np.broadcast_to(density, (n,)))
        m = _i32(np.broadcast_to(materialID, (n,)))
        c = None if clumpID is None else _i32(np.broadcast_to(clumpID, (n,)))
        call("demsph_dem_add_balls", self._h, n, _dp(p), _dp(v), _dp(w), _dp(r), _dp(d), _ip(m), _ip(c), 0)

    def addBall(self, position, velocity, angularVelocity, radius, density, materialID, clumpID=-1):
        self.addBalls([position], [velocity], [angularVelocity], radius, density, materialID, clumpID)

    def addFixedBalls(self, position, radius, materialID, clumpID=None):
        p = _f64(position, (-1, 3))
        n = p.shape[0]
        r = _f64(np.broadcast_to(radius, (n,)))
        m = _i32(np.broadcast_to(materialID, (n,)))
        c = None if clumpID is None else _i32(np.broadcast_to(clumpID, (n,)))
        call("demsph_dem_add_balls", self._h, n, _dp(p), None, None, _dp(r), None, _ip(m), _ip(c), 1)

    def addFixedBall(self, position, radius, materialID, clumpID=-1):
        self.addFixedBalls([position], radius, materialID, clumpID)

    def addClump(self, point, radius, centroidPosition, velocity, angularVelocity, mass, inertiaTensor,
                 materialID):
        p = _f64(point, (-1, 3))
        call("demsph_dem_add_clump", self._h, p.shape[0], _dp(p), _dp(_f64(radius)), _dp(_v3(centroidPosition)),
             _dp(_v3(velocity)), _dp(_v3(angularVelocity)), float(mass), _dp(_f64(inertiaTensor, (6,))),
             int(materialID))

    def addMeshWall(self, vertexPosition, triIndex0, triIndex1, triIndex2, position, velocity=None,
                    angularVelocity=None, materialID=0):
        """Like the reference, velocity / angularVelocity are not applied
        (DEMSolver.h:1901-1911); use setMeshWallMotion."""
        v = _f64(vertexPosition, (-1, 3))
        t0, t1, t2 = _i32(triIndex0), _i32(triIndex1), _i32(triIndex2)
        call("demsph_dem_add_mesh_wall", self._h, v.shape[0], _dp(v), t0.shape[0], _ip(t0), _ip(t1), _ip(t2),
             _dp(_v3(position)), int(materialID))
        self._nvert += v.shape[0]

    def setMeshWallMotion(self, wall, velocity, angularVelocity):
        call("demsph_dem_set_wall_motion", self._h, int(wall), _dp(_v3(velocity)), _dp(_v3(angularVelocity)))

    def addBondedInteraction(self, objectPointed, objectPointing, ballPosition):
        a, b = _i32(objectPointed), _i32(objectPointing)
        p = _f64(ballPosition, (-1, 3))
        call("demsph_dem_add_bonds", self._h, a.shape[0], _ip(a), _ip(b), _dp(p), p.shape[0])

    def setPeriodicBoundary(self, X, Y, Z):
        """setPeriodicBoundary (DEMSolver.h:1944-1959): periodic ghost passes
        along the flagged axes (before initialize)."""
        call("demsph_dem_set_periodic", self._h, int(bool(X)), int(bool(Y)), int(bool(Z)))

    # ------------------------------------------------ external force hook --
    def setConstantForce(self, force, rampTime=0.0):
        f = _f64(force, (-1, 3))
        call("demsph_dem_set_constant_force", self._h, f.shape[0], _dp(f), float(rampTime))

    def setGlobalDamping(self, dampCoeff):
        call("demsph_dem_set_global_damping", self._h, float(dampCoeff))

    def setBuoyancyDrag(self, rhoFluid, Cd, gravity, fluidVelocity, waterLevel):
        call("demsph_dem_set_buoyancy_drag", self._h, float(rhoFluid), float(Cd), _dp(_v3(gravity)),
             _dp(_v3(fluidVelocity)), float(waterLevel))

    # ---------------------------------------------------------------- run --
    def initialize(self, minBoundary, maxBoundary, gravity, timeStep, precision="mixed"):
        prec = _lib.PRECISION_FP64 if precision in ("fp64", _lib.PRECISION_FP64) else _lib.PRECISION_MIXED
        call("demsph_dem_initialize", self._h, _dp(_v3(minBoundary)), _dp(_v3(maxBoundary)), _dp(_v3(gravity)),
             float(timeStep), prec)

    def step(self, numSteps=1):
        call("demsph_dem_step", self._h, int(numSteps))

    def solve(self, minBoundary, maxBoundary, gravity, timeStep, maximumTime, numFrame=0, dir=None,
              deviceID=0, maximumThread=256, precision="mixed"):
        """DEMSolver::solve (DEMSolver.h:1961-2049): initialise, then step to
        maximumTime; with `dir`, VTU frames as the reference writes them
        (frame 0 after initialisation, then every numStep / numFrame steps)."""
        self.initialize(minBoundary, maxBoundary, gravity, timeStep, precision)
        total = num_steps(timeStep, maximumTime)
        if dir is None:
            self.step(total)
            return
        _run_frames(self, total, numFrame, lambda f: self.writeVTU(dir, f))

    def writeVTU(self, dir, frame, what=None):
        """ball / triangleWall / ballInteraction / bondedInteraction /
        ballTriangleInteraction _NNNN.vtu in `dir` (the reference's files)."""
        if what is None:
            what = 1 | 4 | 8 | (2 | 16 if self._has_walls() else 0)
        call("demsph_dem_write_vtu", self._h, str(dir).encode(), int(frame), int(what))

    def _has_walls(self):
        return getattr(self, "_nvert", 0) > 0

    def neighborSearch(self):
        call("demsph_dem_neighbor_search", self._h)

    def calculateBallContactForceTorque(self, timeStep):
        call("demsph_dem_eval_forces", self._h, float(timeStep), 0, 0.0)

    def evalForces(self, timeStep, walls=False, wallTimeStep=0.0, periodic=False, external=False):
        """One force evaluation (calculateBallContactForceTorque, DEMSolver.h:
        599-695) with, optionally, the wall contacts (addTriangleContact-
        ForceTorque(wallTimeStep)), the periodic ghost passes and the external
        forces (the configured hooks and a callback, at the scene's time)."""
        flags = (1 if walls else 0) | (2 if periodic else 0) | (4 if external else 0)
        call("demsph_dem_eval_forces", self._h, float(timeStep), flags, float(wallTimeStep))

    def setExternalHook(self, fn):
        """addExternalForceTorque (virtual, DEMSolver.h:1372) as a Python
        callable fn(iStep, time), called after each force evaluation of a
        step; inside it, hookArrays() gives the ball arrays in the reference's
        layout for launchers such as launchAddConstantForce.  None removes it."""
        if fn is None:
            self._hook = None
            call("demsph_dem_set_external_hook", self._h, _lib.HOOK_FN(), None)
            return
        self._hook = _lib.HOOK_FN(lambda user, iStep, time: fn(int(iStep), float(time)))
        call("demsph_dem_set_external_hook", self._h, self._hook, None)

    def hookArrays(self):
        """demsph_dem_hook_arrays: the device pointers an external-force
        callback works on (current only while it runs)."""
        a = _lib.BallArrays()
        call("demsph_dem_hook_arrays", self._h, C.byref(a))
        return a

    # ------------------------------------------------------------ getters --
    def _n(self, fn, *a):
        n = C.c_long()
        call(fn, self._h, *a, C.byref(n))
        return n.value

    @property
    def numBalls(self):
        return self._n("demsph_dem_num_balls")

    def stepIndex(self):
        s, t = C.c_long(), C.c_double()
        call("demsph_dem_step_index", self._h, C.byref(s), C.byref(t))
        return s.value, t.value

    def getBall(self):
        n = self.numBalls
        out = {k: np.zeros((n, 3)) for k in ("position", "velocity", "angularVelocity", "force", "torque")}
        call("demsph_dem_get_balls", self._h, _dp(out["position"]), _dp(out["velocity"]),
             _dp(out["angularVelocity"]), _dp(out["force"]), _dp(out["torque"]))
        return out

    def setBall(self, position=None, velocity=None, angularVelocity=None):
        n = self.numBalls
        f = lambda x: None if x is None else _f64(x, (n, 3))
        call("demsph_dem_set_balls", self._h, _dp(f(position)), _dp(f(velocity)), _dp(f(angularVelocity)))

    def getPairs(self, which=0):
        """which = 0: ball-ball (getBallPair*), 1: ball-triangle (getBallTrianglePair*)."""
        n = self._n("demsph_dem_num_pairs", which)
        out = {"objectPointed": np.zeros(n, np.int32), "objectPointing": np.zeros(n, np.int32)}
        for k in ("sliding", "rolling", "torsion", "force", "torqueB"):
            out[k] = np.zeros((n, 3))
        call("demsph_dem_get_pairs", self._h, which, _ip(out["objectPointed"]), _ip(out["objectPointing"]),
             _dp(out["sliding"]), _dp(out["rolling"]), _dp(out["torsion"]), _dp(out["force"]), _dp(out["torqueB"]))
        return out

    def getBallPairPointed(self):
        return self.getPairs(0)["objectPointed"]

    def getBallPairPointing(self):
        return self.getPairs(0)["objectPointing"]

    def importSprings(self, objectPointed, objectPointing, sliding, rolling, torsion):
        a, b = _i32(objectPointed), _i32(objectPointing)
        call("demsph_dem_import_springs", self._h, a.shape[0], _ip(a), _ip(b), _dp(_f64(sliding, (-1, 3))),
             _dp(_f64(rolling, (-1, 3))), _dp(_f64(torsion, (-1, 3))))

    def importWallSprings(self, ball, triangle, sliding, rolling, torsion):
        a, b = _i32(ball), _i32(triangle)
        call("demsph_dem_import_wall_springs", self._h, a.shape[0], _ip(a), _ip(b), _dp(_f64(sliding, (-1, 3))),
             _dp(_f64(rolling, (-1, 3))), _dp(_f64(torsion, (-1, 3))))

    def copyMembers(self, source, srcStart, dstStart, num, triDelta, shift):
        """Device-side carry of continuing batch members from `source` (a
        DEMSolver): member k's balls [srcStart[k], +num[k]) there become
        [dstStart[k], ...) here, triangle indices moved by triDelta[k],
        positions by shift[k]."""
        k = len(num)
        call("demsph_dem_copy_members", self._h, source._h, k, _ip(_i32(srcStart)), _ip(_i32(dstStart)),
             _ip(_i32(num)), _ip(_i32(triDelta)), _dp(_f64(shift, (k, 3))))

    def copyMemberBodies(self, source, srcClump, dstClump, numClumps, srcBond, dstBond, numBonds, shift):
        """Device-side carry of continuing members' clumps and bonds from
        `source`, after copyMembers: member k's clumps [srcClump[k],
        +numClumps[k]) and bonds [srcBond[k], +numBonds[k]) there become
        [dstClump[k], ...) and [dstBond[k], ...) here, positions moved by shift[k]."""
        k = len(numClumps)
        call("demsph_dem_copy_member_bodies", self._h, source._h, k, _ip(_i32(srcClump)), _ip(_i32(dstClump)),
             _ip(_i32(numClumps)), _ip(_i32(srcBond)), _ip(_i32(dstBond)), _ip(_i32(numBonds)),
             _dp(_f64(shift, (k, 3))))

    def setGraphs(self, enable=True):
        """Replay the step loop as CUDA graphs (default) or launch directly."""
        call("demsph_dem_set_graphs", self._h, int(bool(enable)))

    def setCellFactor(self, factor):
        """Ball grid cell edge as a multiple of 2 r_max, before initialize (autotuner)."""
        call("demsph_dem_set_cell_factor", self._h, float(factor))

    def reserve(self, pairs=0, reverse=0, triangles=0):
        """Raise the initial list capacities per ball (before initialize)."""
        call("demsph_dem_reserve", self._h, int(pairs), int(reverse), int(triangles))

    def capacity(self):
        k = [C.c_int(), C.c_int(), C.c_int()]
        call("demsph_dem_capacity", self._h, *[C.byref(x) for x in k])
        return tuple(x.value for x in k)

    def assembleBalls(self, members, offsets, matOffsets):
        """Places sealed DEMMember records' balls into this scene (which has
        none yet), member k translated by offsets[k], material ids shifted by
        matOffsets[k]."""
        arr = (C.c_void_p * len(members))(*[m._h.value for m in members])
        call("demsph_dem_assemble_balls", self._h, len(members), arr, _dp(_f64(offsets, (len(members), 3))),
             _ip(_i32(matOffsets)))

    def getBondedInteraction(self):
        n = self._n("demsph_dem_num_bonds")
        out = {"objectPointed": np.zeros(n, np.int32), "objectPointing": np.zeros(n, np.int32),
               "isBonded": np.zeros(n, np.int32), "normalForce": np.zeros(n), "torsionTorque": np.zeros(n)}
        for k in ("shearForce", "bendingTorque", "normal", "point"):
            out[k] = np.zeros((n, 3))
        call("demsph_dem_get_bonds", self._h, _ip(out["objectPointed"]), _ip(out["objectPointing"]),
             _ip(out["isBonded"]), _dp(out["normalForce"]), _dp(out["torsionTorque"]), _dp(out["shearForce"]),
             _dp(out["bendingTorque"]), _dp(out["normal"]), _dp(out["point"]))
        return out

    def diagnostics(self):
        """demsph_dem_diagnostics: FP64 momentum, angular momentum, kinetic
        energies and mass of the moving bodies, and the summed ball force."""
        out = np.zeros(12)
        call("demsph_dem_diagnostics", self._h, _dp(out))
        return {"momentum": out[0:3], "angularMomentum": out[3:6], "kineticEnergy": out[6],
                "rotationalEnergy": out[7], "mass": out[8], "forceSum": out[9:12]}

    def snapshot(self):
        """A device copy of the dynamic state (Snapshot.restore puts it back)."""
        return Snapshot(self, "dem")

    def setBondedInteraction(self, isBonded=None, normalForce=None, torsionTorque=None, shearForce=None,
                             bendingTorque=None, normal=None, point=None):
        """Writes the bond state (getBondedInteraction's order; None keeps a field)."""
        n = self._n("demsph_dem_num_bonds")
        i = lambda x: None if x is None else _i32(x)
        d1 = lambda x: None if x is None else _f64(x, (n,))
        d3 = lambda x: None if x is None else _f64(x, (n, 3))
        ok = i(isBonded)
        call("demsph_dem_set_bonds", self._h, n, _ip(ok), _dp(d1(normalForce)), _dp(d1(torsionTorque)),
             _dp(d3(shearForce)), _dp(d3(bendingTorque)), _dp(d3(normal)), _dp(d3(point)))

    def getClump(self):
        n = self._n("demsph_dem_num_clumps")
        out = {"position": np.zeros((n, 3)), "velocity": np.zeros((n, 3)), "angularVelocity": np.zeros((n, 3)),
               "orientation": np.zeros((n, 4))}
        if n:
            call("demsph_dem_get_clumps", self._h, _dp(out["position"]), _dp(out["velocity"]),
                 _dp(out["angularVelocity"]), _dp(out["orientation"]))
        return out

    def getMeshWall(self, numWalls=1):
        out = {"position": np.zeros((numWalls, 3)), "orientation": np.zeros((numWalls, 4)),
               "vertexGlobal": np.zeros((self._nvert, 3))}
        call("demsph_dem_get_walls", self._h, _dp(out["position"]), _dp(out["orientation"]),
             _dp(out["vertexGlobal"]))
        return out


class SPHMember:
    """One scene's fluid and dummy particles held on the device, from which
    batch scenes are assembled (WCSPHSolver.assemble)."""

    def __init__(self, stream=None):
        self._h = C.c_void_p()
        call("demsph_sph_member_create", C.byref(self._h), _stream_ptr(stream))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().demsph_sph_member_destroy(h)
            except Exception:
                pass
            self._h = None

    def _add(self, dummy, position, velocity, soundSpeed, spacing, density, viscosity):
        p = _f64(position, (-1, 3))
        n = p.shape[0]
        v = None if velocity is None else _f64(velocity, (n, 3))
        b = lambda x: _f64(np.broadcast_to(x, (n,)))
        call("demsph_sph_member_add", self._h, int(dummy), n, _dp(p), _dp(v), _dp(b(soundSpeed)), _dp(b(spacing)),
             _dp(b(density)), _dp(b(viscosity)))

    def addSPHs(self, position, velocity, soundSpeed, spacing, density, viscosity):
        self._add(0, position, velocity, soundSpeed, spacing, density, viscosity)

    def addDummies(self, position, velocity, soundSpeed, spacing, density, viscosity):
        self._add(1, position, velocity, soundSpeed, spacing, density, viscosity)

    def seal(self):
        call("demsph_sph_member_seal", self._h)
        return self

    def num(self, dummy=False):
        n = C.c_long()
        call("demsph_sph_member_count", self._h, int(dummy), C.byref(n))
        return n.value


class WCSPHSolver:
    """Weakly compressible SPH with fixed dummy wall particles."""

    def __init__(self, stream=None):
        self._h = C.c_void_p()
        call("demsph_sph_create", C.byref(self._h), _stream_ptr(stream))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().demsph_sph_destroy(h)
            except Exception:
                pass
            self._h = None

    def _add(self, dummy, position, velocity, soundSpeed, spacing, density, viscosity):
        p = _f64(position, (-1, 3))
        n = p.shape[0]
        v = None if velocity is None else _f64(velocity, (n, 3))
        b = lambda x: _f64(np.broadcast_to(x, (n,)))
        call("demsph_sph_add", self._h, int(dummy), n, _dp(p), _dp(v), _dp(b(soundSpeed)), _dp(b(spacing)),
             _dp(b(density)), _dp(b(viscosity)))

    def addSPHs(self, position, velocity, soundSpeed, spacing, density, viscosity):
        self._add(0, position, velocity, soundSpeed, spacing, density, viscosity)

    def addDummies(self, position, velocity, soundSpeed, spacing, density, viscosity):
        self._add(1, position, velocity, soundSpeed, spacing, density, viscosity)

    def addSPH(self, position, velocity, soundSpeed, spacing, density, viscosity):
        self._add(0, [position], [velocity], soundSpeed, spacing, density, viscosity)

    def addDummy(self, position, velocity, soundSpeed, spacing, density, viscosity):
        self._add(1, [position], [velocity], soundSpeed, spacing, density, viscosity)

    def initialize(self, minBoundary, maxBoundary, gravity, timeStep, precision="fp64"):
        prec = _lib.PRECISION_MIXED if precision in ("mixed", _lib.PRECISION_MIXED) else _lib.PRECISION_FP64
        call("demsph_sph_initialize", self._h, _dp(_v3(minBoundary)), _dp(_v3(maxBoundary)), _dp(_v3(gravity)),
             float(timeStep), prec)

    def step(self, numSteps=1):
        """Queues numSteps steps on the scene's stream and returns (getters
        and synchronize() wait for them)."""
        call("demsph_sph_step", self._h, int(numSteps))

    def synchronize(self):
        """Waits for the scene's queued steps."""
        call("demsph_sph_synchronize", self._h)

    def solve(self, minBoundary, maxBoundary, gravity, timeStep, maximumTime, numFrame=0, dir=None, deviceID=0,
              maximumThread=256, precision="fp64"):
        """WCSPHSolver::solve (WCSPHSolver.h:567-624), with VTU frames in
        `dir` as the reference writes them."""
        self.initialize(minBoundary, maxBoundary, gravity, timeStep, precision)
        total = num_steps(timeStep, maximumTime)
        if dir is None:
            self.step(total)
            return
        _run_frames(self, total, numFrame, lambda f: self.writeVTU(dir, f))

    def writeVTU(self, dir, frame, what=3):
        """SPH_NNNN.vtu and dummy_NNNN.vtu in `dir` (the reference's files)."""
        call("demsph_sph_write_vtu", self._h, str(dir).encode(), int(frame), int(what))

    def neighborSearch(self):
        call("demsph_sph_neighbor_search", self._h)

    def evalAcceleration(self):
        call("demsph_sph_eval_accel", self._h)

    def num(self, dummy=False):
        n = C.c_long()
        call("demsph_sph_num", self._h, int(dummy), C.byref(n))
        return n.value

    def stepIndex(self):
        s, t = C.c_long(), C.c_double()
        call("demsph_sph_step_index", self._h, C.byref(s), C.byref(t))
        return s.value, t.value

    def _get(self, dummy):
        n = self.num(dummy)
        out = {"position": np.empty((n, 3)), "velocity": np.empty((n, 3)), "acceleration": np.empty((n, 3)),
               "density": np.empty(n), "pressure": np.empty(n), "densityChange": np.empty(n),
               "normal": np.empty((n, 3))}
        call("demsph_sph_get", self._h, int(dummy), _dp(out["position"]), _dp(out["velocity"]),
             _dp(out["acceleration"]), _dp(out["density"]), _dp(out["pressure"]), _dp(out["densityChange"]),
             _dp(out["normal"]))
        return out

    def snapshot(self):
        """A device copy of the fluid's state (Snapshot.restore puts it back)."""
        return Snapshot(self, "sph")

    def setUniformKernels(self, enable=True):
        """Use (default) or not the passes specialised for uniform particle
        constants (mixed precision)."""
        call("demsph_sph_set_uniform_kernels", self._h, int(bool(enable)))

    def uniformKernels(self):
        """Whether the specialised mixed-precision passes are in use."""
        a = C.c_int()
        call("demsph_sph_uniform_kernels", self._h, C.byref(a))
        return bool(a.value)

    def diagnostics(self):
        """demsph_sph_diagnostics: FP64 mass, momentum, kinetic and potential
        energy, summed density change and volume of the fluid."""
        out = np.zeros(8)
        call("demsph_sph_diagnostics", self._h, _dp(out))
        return {"mass": out[0], "momentum": out[1:4], "kineticEnergy": out[4], "potentialEnergy": out[5],
                "densityChangeSum": out[6], "volume": out[7]}

    def getSPH(self):
        return self._get(False)

    def getDummy(self):
        return self._get(True)

    def setSPH(self, position=None, velocity=None, density=None, pressure=None, densityChange=None):
        n = self.num()
        f = lambda x, s: None if x is None else _f64(x, s)
        call("demsph_sph_set", self._h, _dp(f(position, (n, 3))), _dp(f(velocity, (n, 3))), _dp(f(density, (n,))),
             _dp(f(pressure, (n,))), _dp(f(densityChange, (n,))))

    def assemble(self, members, offsets, minBoundary, maxBoundary, gravity, timeStep, precision="mixed"):
        """Initialises this (empty) scene on the device from sealed
        SPHMember records, member k translated by offsets[k]."""
        arr = (C.c_void_p * len(members))(*[m._h.value for m in members])
        off = _f64(offsets, (len(members), 3))
        prec = _lib.PRECISION_MIXED if precision in ("mixed", _lib.PRECISION_MIXED) else _lib.PRECISION_FP64
        call("demsph_sph_assemble", self._h, len(members), arr, _dp(off), _dp(_v3(minBoundary)),
             _dp(_v3(maxBoundary)), _dp(_v3(gravity)), float(timeStep), prec)

    def setGraphs(self, enable=True):
        """Replay the step loop as CUDA graphs (default) or launch directly."""
        call("demsph_sph_set_graphs", self._h, int(bool(enable)))

    def tune(self, trials=5):
        """Autotunes the neighbour-list build's block shape on the current
        state; returns (chosen shape, milliseconds per build of each shape)."""
        ns = _lib.lib().demsph_sph_num_list_shapes()
        ms = np.zeros(ns)
        ch = C.c_int()
        call("demsph_sph_tune", self._h, int(trials), C.byref(ch), _dp(ms))
        return ch.value, ms

    def setSkin(self, fraction):
        """Skin of the neighbour rows as a fraction of 2 h_max (0: exact lists
        rebuilt every step); before initialize() it also sizes the grid."""
        call("demsph_sph_set_skin", self._h, float(fraction))

    def tuneSkin(self, steps=20):
        """Times `steps` steps with no skin, half the grid's and the grid's
        skin from the same state (restored after) and keeps the fastest;
        returns (chosen fraction, [ms per step for each])."""
        c = C.c_double()
        ms = np.zeros(3)
        call("demsph_sph_tune_skin", self._h, int(steps), C.byref(c), _dp(ms))
        return c.value, list(ms)

    def skinStats(self):
        """(fraction in use, rebuilds so far)."""
        f, r = C.c_double(), C.c_long()
        call("demsph_sph_skin_stats", self._h, C.byref(f), C.byref(r))
        return f.value, r.value

    def setListShape(self, shape):
        call("demsph_sph_set_list_shape", self._h, int(shape))

    def setConditionalRebuild(self, enable=True):
        """Graph steps skip the list rebuild's launches through a conditional
        node, or launch them gated every step (the default, which profilers
        can see); same results."""
        call("demsph_sph_set_conditional_rebuild", self._h, int(bool(enable)))

    def conditionalRebuild(self):
        """(in use, kernels one rebuild runs)."""
        a, n = C.c_int(), C.c_long()
        call("demsph_sph_conditional_rebuild", self._h, C.byref(a), C.byref(n))
        return bool(a.value), n.value

    def setCellFactor(self, factor):
        """Grid cell edge as a multiple of 2 h_max (1 + skin), before initialize (autotuner)."""
        call("demsph_sph_set_cell_factor", self._h, float(factor))

    def setListHeadroom(self, fraction):
        """Row capacity above the initial longest row, before initialize (autotuner)."""
        call("demsph_sph_set_list_headroom", self._h, float(fraction))

    def listCapacity(self):
        """(fluid-fluid, fluid-dummy) row capacities."""
        a, b = C.c_int(), C.c_int()
        call("demsph_sph_list_capacity", self._h, C.byref(a), C.byref(b))
        return a.value, b.value

    def copyMembers(self, source, srcStart, dstStart, num, shift):
        """Device-side carry of fluid state from `source` (a WCSPHSolver):
        member k's caller ids [srcStart[k], +num[k]) there are
        [dstStart[k], ...) here, positions moved by shift[k]."""
        k = len(num)
        call("demsph_sph_copy_members", self._h, source._h, k, _ip(_i32(srcStart)), _ip(_i32(dstStart)),
             _ip(_i32(num)), _dp(_f64(shift, (k, 3))))

    def getPairs(self, which=0):
        """which = 0 fluid-fluid, 1 fluid-dummy, 2 dummy-dummy; original indices, CSR order."""
        n = C.c_long()
        call("demsph_sph_num_pairs", self._h, int(which), C.byref(n))
        a, b = np.zeros(n.value, np.int32), np.zeros(n.value, np.int32)
        call("demsph_sph_get_pairs", self._h, int(which), _ip(a), _ip(b))
        return a, b


class DEMSPHCoupling:
    """Particle-level two-way coupling of DEM balls and a WCSPH fluid.

    The reference couples balls to a fluid only through the buoyancy-drag
    plane of DEMSolver.setBuoyancyDrag (externalForceTorque.cu:66-133).  Here
    each coupled ball is sampled by markers -- moving boundary particles on
    shells inside its surface -- that act on the fluid exactly as the
    reference's dummy particles do (WCSPHIntegrationKernel.cu:110-143,
    240-270), with the ball's rigid velocity and an outward normal; the ball
    receives minus the sum of m_a times its markers' terms in the fluid
    accelerations as force, and offset x force as torque.

    Both solvers must be initialised; the DEM time step times demSubsteps
    must equal the fluid's.
    """

    def __init__(self, sph: WCSPHSolver, dem: DEMSolver):
        self.sph = sph
        self.dem = dem

    def addBalls(self, balls, spacing, smoothingLength, soundSpeed, viscosity, density):
        """Couples DEM balls `balls` (indices) with markers of the given
        spacing, h, sound speed, viscosity and rest density."""
        b = _i32(np.atleast_1d(balls))
        call("demsph_sph_couple_balls", self.sph._h, self.dem._h, len(b), _ip(b), float(spacing),
             float(smoothingLength), float(soundSpeed), float(viscosity), float(density))

    def step(self, numSteps=1, demSubsteps=1):
        call("demsph_sph_couple_step", self.sph._h, self.dem._h, int(numSteps), int(demSubsteps))

    def numMarkers(self):
        n, b = C.c_long(), C.c_long()
        call("demsph_sph_num_markers", self.sph._h, C.byref(n), C.byref(b))
        return n.value, b.value

    def getMarkers(self):
        """Per marker (body order): position, velocity, normal, last reaction, ball."""
        n, _ = self.numMarkers()
        out = {"position": np.zeros((n, 3)), "velocity": np.zeros((n, 3)), "normal": np.zeros((n, 3)),
               "force": np.zeros((n, 3)), "ball": np.zeros(n, np.int32)}
        call("demsph_sph_get_markers", self.sph._h, _dp(out["position"]), _dp(out["velocity"]),
             _dp(out["normal"]), _dp(out["force"]), _ip(out["ball"]))
        return out

    def getForces(self):
        """(ball indices, force (n, 3), torque (n, 3)) on the coupled balls."""
        _, nb = self.numMarkers()
        ball = np.zeros(nb, np.int32)
        F, T = np.zeros((nb, 3)), np.zeros((nb, 3))
        call("demsph_sph_get_coupling", self.sph._h, _ip(ball), _dp(F), _dp(T))
        return ball, F, T


class Snapshot:
    """A device copy of a scene's dynamic state (demsph_dem_snapshot /
    demsph_sph_snapshot); restore() puts it back into the same scene."""

    def __init__(self, solver, kind):
        self._solver, self._kind = solver, kind
        self._h = C.c_void_p()
        call(f"demsph_{kind}_snapshot", solver._h, C.byref(self._h))

    def restore(self):
        call(f"demsph_{self._kind}_restore", self._solver._h, self._h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                getattr(_lib.lib(), f"demsph_{self._kind}_snapshot_destroy")(h)
            except Exception:
                pass
            self._h = None
