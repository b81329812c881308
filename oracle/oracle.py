"""ctypes wrapper of the FP64 CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
load this module.  The product package never imports it.

The classes mirror the reference's host API: ``OracleDEM`` follows
``DEMSolver`` (DEMSPH/kernel/DEMSolver.h:1633-1961) and ``OracleSPH`` follows
``WCSPHSolver`` (DEMSPH/kernel/WCSPHSolver.h:522-624).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libdemsph_oracle.so")
_lib = None

_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int)
_vp = C.c_void_p


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        sig = {
            "oracle_num_threads": (C.c_int, [C.c_int]),
            "oracle_dem_create": (_vp, []),
            "oracle_dem_destroy": (None, [_vp]),
            "oracle_dem_set_hertzian_pair": (None, [_vp, C.c_int, C.c_int] + [C.c_double] * 8),
            "oracle_dem_set_linear_pair": (None, [_vp, C.c_int, C.c_int] + [C.c_double] * 11),
            "oracle_dem_set_bonded_pair": (None, [_vp, C.c_int, C.c_int] + [C.c_double] * 6),
            "oracle_dem_add_balls": (None, [_vp, C.c_long, _d, _d, _d, _d, _d, _i, _i, C.c_int]),
            "oracle_dem_add_clump": (None, [_vp, C.c_long, _d, _d, _d, _d, _d, C.c_double, _d, C.c_int]),
            "oracle_dem_add_mesh_wall": (None, [_vp, C.c_long, _d, C.c_long, _i, _i, _i, _d, C.c_int]),
            "oracle_dem_set_wall_motion": (None, [_vp, C.c_int, _d, _d]),
            "oracle_dem_add_bonds": (None, [_vp, C.c_long, _i, _i, _d, C.c_long]),
            "oracle_dem_set_buoyancy_drag": (None, [_vp, C.c_double, C.c_double, _d, _d, C.c_double]),
            "oracle_dem_set_global_damping": (None, [_vp, C.c_double]),
            "oracle_dem_set_constant_force": (None, [_vp, C.c_long, _d, C.c_double]),
            "oracle_dem_initialize": (C.c_int, [_vp, _d, _d, _d, C.c_double]),
            "oracle_dem_step": (C.c_int, [_vp, C.c_long]),
            "oracle_dem_neighbor_search": (None, [_vp]),
            "oracle_dem_eval_forces": (None, [_vp, C.c_double, C.c_int, C.c_double]),
            "oracle_dem_num_balls": (C.c_long, [_vp]),
            "oracle_dem_num_pairs": (C.c_long, [_vp]),
            "oracle_dem_num_wall_pairs": (C.c_long, [_vp]),
            "oracle_dem_num_bonds": (C.c_long, [_vp]),
            "oracle_dem_step_index": (C.c_long, [_vp]),
            "oracle_dem_get_balls": (None, [_vp, _d, _d, _d, _d, _d]),
            "oracle_dem_set_balls": (None, [_vp, _d, _d, _d]),
            "oracle_dem_get_pairs": (None, [_vp, C.c_int, _i, _i, _d, _d, _d, _d, _d, _d, _d]),
            "oracle_dem_set_periodic": (None, [_vp, C.c_int, C.c_int, C.c_int]),
            "oracle_dem_num_ghost_pairs": (C.c_long, [_vp, C.c_int]),
            "oracle_dem_get_ghost_pairs": (None, [_vp, C.c_int, _i, _i, _d, _d]),
            "oracle_dem_import_springs": (None, [_vp, C.c_long, _i, _i, _d, _d, _d]),
            "oracle_dem_get_bonds": (None, [_vp, _i, _i, _i, _d, _d, _d, _d, _d, _d]),
            "oracle_dem_num_clumps": (C.c_long, [_vp]),
            "oracle_dem_get_clumps": (None, [_vp, _d, _d, _d, _d]),
            "oracle_dem_num_walls": (C.c_long, [_vp]),
            "oracle_dem_get_walls": (None, [_vp, _d, _d, _d]),
            "oracle_sph_create": (_vp, []),
            "oracle_sph_destroy": (None, [_vp]),
            "oracle_sph_add": (None, [_vp, C.c_int, C.c_long, _d, _d, _d, _d, _d, _d]),
            "oracle_sph_initialize": (C.c_int, [_vp, _d, _d, _d, C.c_double]),
            "oracle_sph_step": (C.c_int, [_vp, C.c_long]),
            "oracle_sph_neighbor_search": (None, [_vp]),
            "oracle_sph_eval_accel": (None, [_vp]),
            "oracle_sph_eval_density": (None, [_vp, C.c_double]),
            "oracle_sph_num": (C.c_long, [_vp, C.c_int]),
            "oracle_sph_num_pairs": (C.c_long, [_vp, C.c_int]),
            "oracle_sph_get_pairs": (None, [_vp, C.c_int, _i, _i]),
            "oracle_sph_get": (None, [_vp, C.c_int, _d, _d, _d, _d, _d, _d, _d]),
            "oracle_sph_set": (None, [_vp, _d, _d, _d, _d, _d]),
            "oracle_sph_couple_balls": (C.c_int, [_vp, _vp, C.c_long, _i, C.c_double, C.c_double, C.c_double,
                                                  C.c_double, C.c_double]),
            "oracle_couple_step": (C.c_int, [_vp, _vp, C.c_long, C.c_int]),
            "oracle_sph_num_markers": (C.c_long, [_vp]),
            "oracle_sph_get_markers": (None, [_vp, _d, _d, _d, _d, _i]),
            "oracle_sph_get_coupling": (None, [_vp, _vp, _i, _d, _d]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _dp(a):
    if a is None:
        return None
    return a.ctypes.data_as(_d)


def _ip(a):
    if a is None:
        return None
    return a.ctypes.data_as(_i)


def _f64(a, shape=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if shape is not None:
        a = a.reshape(shape)
    return a


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def set_threads(n=0):
    return lib().oracle_num_threads(int(n))


class OracleDEM:
    """FP64 restatement of DEMSolver (DEMSPH/kernel/DEMSolver.h:144-2078)."""

    def __init__(self):
        self._L = lib()
        self.h = self._L.oracle_dem_create()

    def __del__(self):
        try:
            self._L.oracle_dem_destroy(self.h)
        except Exception:
            pass

    def set_hertzian_pair(self, a, b, E, G, e, krks=0.0, ktks=0.0, mus=0.0, mur=0.0, mut=0.0):
        self._L.oracle_dem_set_hertzian_pair(self.h, a, b, E, G, e, krks, ktks, mus, mur, mut)

    def set_linear_pair(self, a, b, kn, ks, kr, kt, dn, ds, dr, dt, mus, mur, mut):
        self._L.oracle_dem_set_linear_pair(self.h, a, b, kn, ks, kr, kt, dn, ds, dr, dt, mus, mur, mut)

    def set_bonded_pair(self, a, b, gamma, Eb, knks, sigma, C_, mu):
        self._L.oracle_dem_set_bonded_pair(self.h, a, b, gamma, Eb, knks, sigma, C_, mu)

    def add_balls(self, pos, vel, angvel, radius, density, material, clump=None, fixed=False):
        pos = _f64(pos, (-1, 3))
        n = pos.shape[0]
        vel = _f64(vel if vel is not None else np.zeros((n, 3)), (-1, 3))
        w = _f64(angvel if angvel is not None else np.zeros((n, 3)), (-1, 3))
        rad = _f64(np.broadcast_to(radius, (n,)))
        den = _f64(np.broadcast_to(density if density is not None else 0.0, (n,)))
        mat = _i32(np.broadcast_to(material, (n,)))
        cl = _i32(np.broadcast_to(-1 if clump is None else clump, (n,)))
        self._L.oracle_dem_add_balls(self.h, n, _dp(pos), _dp(vel), _dp(w), _dp(rad), _dp(den), _ip(mat), _ip(cl),
                                     int(bool(fixed)))

    def add_clump(self, points, radius, centroid, vel, angvel, mass, inertia, material):
        pts = _f64(points, (-1, 3))
        rad = _f64(radius)
        self._L.oracle_dem_add_clump(self.h, pts.shape[0], _dp(pts), _dp(rad), _dp(_f64(centroid)), _dp(_f64(vel)),
                                     _dp(_f64(angvel)), float(mass), _dp(_f64(inertia)), int(material))

    def add_mesh_wall(self, vertices, tri0, tri1, tri2, position, material):
        v = _f64(vertices, (-1, 3))
        t0, t1, t2 = _i32(tri0), _i32(tri1), _i32(tri2)
        self._L.oracle_dem_add_mesh_wall(self.h, v.shape[0], _dp(v), t0.shape[0], _ip(t0), _ip(t1), _ip(t2),
                                         _dp(_f64(position)), int(material))

    def set_wall_motion(self, wall, vel, angvel):
        self._L.oracle_dem_set_wall_motion(self.h, wall, _dp(_f64(vel)), _dp(_f64(angvel)))

    def add_bonds(self, a, b, positions):
        a, b = _i32(a), _i32(b)
        p = _f64(positions, (-1, 3))
        self._L.oracle_dem_add_bonds(self.h, a.shape[0], _ip(a), _ip(b), _dp(p), p.shape[0])

    def set_buoyancy_drag(self, rho, Cd, g, u, level):
        self._L.oracle_dem_set_buoyancy_drag(self.h, rho, Cd, _dp(_f64(g)), _dp(_f64(u)), level)

    def set_global_damping(self, c):
        self._L.oracle_dem_set_global_damping(self.h, c)

    def set_constant_force(self, f, ramp=0.0):
        f = _f64(f, (-1, 3))
        self._L.oracle_dem_set_constant_force(self.h, f.shape[0], _dp(f), ramp)

    def initialize(self, mn, mx, g, dt):
        rc = self._L.oracle_dem_initialize(self.h, _dp(_f64(mn)), _dp(_f64(mx)), _dp(_f64(g)), float(dt))
        if rc != 0:
            raise RuntimeError(f"oracle_dem_initialize failed with status {rc}")

    def step(self, n=1):
        rc = self._L.oracle_dem_step(self.h, int(n))
        if rc != 0:
            raise RuntimeError(f"oracle_dem_step failed with status {rc}")

    def neighbor_search(self):
        self._L.oracle_dem_neighbor_search(self.h)

    def eval_forces(self, dt, walls=False, dt_wall=0.0):
        self._L.oracle_dem_eval_forces(self.h, dt, int(walls), dt_wall)

    @property
    def num_balls(self):
        return self._L.oracle_dem_num_balls(self.h)

    @property
    def step_index(self):
        return self._L.oracle_dem_step_index(self.h)

    def balls(self):
        n = self.num_balls
        out = {k: np.zeros((n, 3)) for k in ("pos", "vel", "angvel", "force", "torque")}
        self._L.oracle_dem_get_balls(self.h, _dp(out["pos"]), _dp(out["vel"]), _dp(out["angvel"]),
                                     _dp(out["force"]), _dp(out["torque"]))
        return out

    def set_balls(self, pos=None, vel=None, angvel=None):
        n = self.num_balls
        p = None if pos is None else _f64(pos, (n, 3))
        v = None if vel is None else _f64(vel, (n, 3))
        w = None if angvel is None else _f64(angvel, (n, 3))
        self._L.oracle_dem_set_balls(self.h, _dp(p), _dp(v), _dp(w))

    def pairs(self, which=0):
        n = self._L.oracle_dem_num_pairs(self.h) if which == 0 else self._L.oracle_dem_num_wall_pairs(self.h)
        out = {"a": np.zeros(n, np.int32), "b": np.zeros(n, np.int32)}
        for k in ("sliding", "rolling", "torsion", "force", "torque", "point"):
            out[k] = np.zeros((n, 3))
        out["overlap"] = np.zeros(n)
        self._L.oracle_dem_get_pairs(self.h, which, _ip(out["a"]), _ip(out["b"]), _dp(out["sliding"]),
                                     _dp(out["rolling"]), _dp(out["torsion"]), _dp(out["force"]),
                                     _dp(out["torque"]), _dp(out["point"]), _dp(out["overlap"]))
        return out

    def set_periodic(self, x, y, z):
        self._L.oracle_dem_set_periodic(self.h, int(bool(x)), int(bool(y)), int(bool(z)))

    def ghost_pairs(self, ghost_set):
        n = self._L.oracle_dem_num_ghost_pairs(self.h, int(ghost_set))
        out = {"a": np.zeros(n, np.int32), "b": np.zeros(n, np.int32), "sliding": np.zeros((n, 3)),
               "force": np.zeros((n, 3))}
        self._L.oracle_dem_get_ghost_pairs(self.h, int(ghost_set), _ip(out["a"]), _ip(out["b"]),
                                           _dp(out["sliding"]), _dp(out["force"]))
        return out

    def import_springs(self, a, b, sliding, rolling, torsion):
        a, b = _i32(a), _i32(b)
        self._L.oracle_dem_import_springs(self.h, a.shape[0], _ip(a), _ip(b), _dp(_f64(sliding, (-1, 3))),
                                          _dp(_f64(rolling, (-1, 3))), _dp(_f64(torsion, (-1, 3))))

    def bonds(self):
        n = self._L.oracle_dem_num_bonds(self.h)
        out = {"a": np.zeros(n, np.int32), "b": np.zeros(n, np.int32), "ok": np.zeros(n, np.int32),
               "normal_force": np.zeros(n), "torsion_torque": np.zeros(n)}
        for k in ("shear_force", "bending_torque", "normal", "point"):
            out[k] = np.zeros((n, 3))
        self._L.oracle_dem_get_bonds(self.h, _ip(out["a"]), _ip(out["b"]), _ip(out["ok"]), _dp(out["normal_force"]),
                                     _dp(out["torsion_torque"]), _dp(out["shear_force"]), _dp(out["bending_torque"]),
                                     _dp(out["normal"]), _dp(out["point"]))
        return out

    def clumps(self):
        n = self._L.oracle_dem_num_clumps(self.h)
        out = {"pos": np.zeros((n, 3)), "vel": np.zeros((n, 3)), "angvel": np.zeros((n, 3)), "q": np.zeros((n, 4))}
        self._L.oracle_dem_get_clumps(self.h, _dp(out["pos"]), _dp(out["vel"]), _dp(out["angvel"]), _dp(out["q"]))
        return out

    def walls(self, num_vertices):
        n = self._L.oracle_dem_num_walls(self.h)
        out = {"pos": np.zeros((n, 3)), "q": np.zeros((n, 4)), "vertices": np.zeros((num_vertices, 3))}
        self._L.oracle_dem_get_walls(self.h, _dp(out["pos"]), _dp(out["q"]), _dp(out["vertices"]))
        return out


class OracleSPH:
    """FP64 restatement of WCSPHSolver (DEMSPH/kernel/WCSPHSolver.h:18-635)."""

    def __init__(self):
        self._L = lib()
        self.h = self._L.oracle_sph_create()

    def __del__(self):
        try:
            self._L.oracle_sph_destroy(self.h)
        except Exception:
            pass

    def _add(self, dummy, pos, vel, c, spacing, density, viscosity):
        pos = _f64(pos, (-1, 3))
        n = pos.shape[0]
        vel = _f64(vel if vel is not None else np.zeros((n, 3)), (-1, 3))
        b = lambda x: _f64(np.broadcast_to(x, (n,)))
        self._L.oracle_sph_add(self.h, int(dummy), n, _dp(pos), _dp(vel), _dp(b(c)), _dp(b(spacing)),
                               _dp(b(density)), _dp(b(viscosity)))

    def add_sph(self, pos, vel, c, spacing, density, viscosity):
        self._add(0, pos, vel, c, spacing, density, viscosity)

    def add_dummy(self, pos, vel, c, spacing, density, viscosity):
        self._add(1, pos, vel, c, spacing, density, viscosity)

    def initialize(self, mn, mx, g, dt):
        rc = self._L.oracle_sph_initialize(self.h, _dp(_f64(mn)), _dp(_f64(mx)), _dp(_f64(g)), float(dt))
        if rc != 0:
            raise RuntimeError(f"oracle_sph_initialize failed with status {rc}")

    def step(self, n=1):
        rc = self._L.oracle_sph_step(self.h, int(n))
        if rc != 0:
            raise RuntimeError(f"oracle_sph_step failed with status {rc}")

    def neighbor_search(self):
        self._L.oracle_sph_neighbor_search(self.h)

    def eval_accel(self):
        self._L.oracle_sph_eval_accel(self.h)

    def eval_density(self, dt):
        self._L.oracle_sph_eval_density(self.h, dt)

    def num(self, dummy=False):
        return self._L.oracle_sph_num(self.h, int(dummy))

    def pairs(self, which=0):
        n = self._L.oracle_sph_num_pairs(self.h, which)
        a, b = np.zeros(n, np.int32), np.zeros(n, np.int32)
        self._L.oracle_sph_get_pairs(self.h, which, _ip(a), _ip(b))
        return a, b

    def state(self, dummy=False):
        n = self.num(dummy)
        out = {"pos": np.zeros((n, 3)), "vel": np.zeros((n, 3)), "acc": np.zeros((n, 3)), "rho": np.zeros(n),
               "p": np.zeros(n), "drho": np.zeros(n), "normal": np.zeros((n, 3))}
        self._L.oracle_sph_get(self.h, int(dummy), _dp(out["pos"]), _dp(out["vel"]), _dp(out["acc"]),
                               _dp(out["rho"]), _dp(out["p"]), _dp(out["drho"]), _dp(out["normal"]))
        return out

    def set_state(self, pos=None, vel=None, rho=None, p=None, drho=None):
        n = self.num()
        f = lambda x, s: None if x is None else _f64(x, s)
        self._L.oracle_sph_set(self.h, _dp(f(pos, (n, 3))), _dp(f(vel, (n, 3))), _dp(f(rho, (n,))),
                               _dp(f(p, (n,))), _dp(f(drho, (n,))))

    # particle-level coupling to DEM balls (no reference counterpart)
    def couple_balls(self, dem, balls, spacing, h, c, nu, rho0):
        balls = np.ascontiguousarray(balls, np.int32)
        rc = self._L.oracle_sph_couple_balls(self.h, dem.h, len(balls), _ip(balls), float(spacing), float(h),
                                             float(c), float(nu), float(rho0))
        if rc != 0:
            raise RuntimeError(f"oracle_sph_couple_balls failed with status {rc}")
        self._dem = dem

    def couple_step(self, dem, n=1, dem_substeps=1):
        rc = self._L.oracle_couple_step(self.h, dem.h, int(n), int(dem_substeps))
        if rc != 0:
            raise RuntimeError(f"oracle_couple_step failed with status {rc}")

    def markers(self):
        n = self._L.oracle_sph_num_markers(self.h)
        out = {"pos": np.zeros((n, 3)), "vel": np.zeros((n, 3)), "normal": np.zeros((n, 3)),
               "force": np.zeros((n, 3)), "ball": np.zeros(n, np.int32)}
        self._L.oracle_sph_get_markers(self.h, _dp(out["pos"]), _dp(out["vel"]), _dp(out["normal"]),
                                       _dp(out["force"]), _ip(out["ball"]))
        return out

    def coupling(self, dem, nbodies):
        ball = np.zeros(nbodies, np.int32)
        F, T = np.zeros((nbodies, 3)), np.zeros((nbodies, 3))
        self._L.oracle_sph_get_coupling(self.h, dem.h, _ip(ball), _dp(F), _dp(T))
        return ball, F, T
