"""Shared test helpers: load a scene into the oracle, compare pair sets and
force fields."""
import numpy as np

from oracle.oracle import OracleDEM, OracleSPH


def oracle_dem(scene):
    o = OracleDEM()
    for r in scene.hertz:
        o.set_hertzian_pair(*r)
    for r in scene.linear:
        o.set_linear_pair(*r)
    for r in scene.bonded:
        o.set_bonded_pair(*r)
    n = scene.position.shape[0]
    fixed = np.zeros(n, bool) if scene.fixed is None else scene.fixed
    starts = np.flatnonzero(np.diff(np.r_[-1, fixed.astype(int)]) != 0)
    bounds = list(starts) + [n]
    w = getattr(scene, "angvel", None)
    for a, b in zip(bounds[:-1], bounds[1:]):
        sl = slice(a, b)
        vel = None if scene.velocity is None else scene.velocity[sl]
        o.add_balls(scene.position[sl], vel, None if w is None else w[sl], scene.radius[sl], scene.density[sl],
                    scene.material[sl], None, fixed=bool(fixed[a]))
    for c in scene.clumps:
        o.add_clump(c["point"], c["radius"], c["centroid"], c["velocity"], c["angularVelocity"], c["mass"],
                    c["inertia"], c["material"])
    for k, wl in enumerate(scene.walls):
        o.add_mesh_wall(wl["vertices"], wl["tri0"], wl["tri1"], wl["tri2"], wl["position"], wl["material"])
        if "velocity" in wl:
            o.set_wall_motion(k, wl["velocity"], wl.get("angularVelocity", (0, 0, 0)))
    if scene.buoyancy is not None:
        o.set_buoyancy_drag(*scene.buoyancy)
    if getattr(scene, "periodic", None) is not None:
        o.set_periodic(*scene.periodic)
    o.initialize(scene.minb, scene.maxb, scene.gravity, scene.dt)
    if scene.bond_initial_contacts:
        p = o.pairs(0)
        o.add_bonds(p["a"], p["b"], scene.position)
    return o


def oracle_sph(scene):
    o = OracleSPH()
    o.add_sph(scene.fluid, None, scene.sound_speed, scene.spacing, scene.density, scene.viscosity)
    o.add_dummy(scene.dummy, None, scene.sound_speed, scene.spacing, scene.density, scene.viscosity)
    o.initialize(scene.minb, scene.maxb, scene.gravity, scene.dt)
    return o


def pair_keys(a, b):
    return np.asarray(a, np.int64) * (1 << 32) + np.asarray(b, np.int64)


def rel_err(x, ref):
    """||x - ref||_2 / ||ref||_2 over all entries (0 when both vanish)."""
    d = np.linalg.norm(np.asarray(x) - np.asarray(ref))
    n = np.linalg.norm(ref)
    return d / n if n > 0 else d


def torque_err(T, T64, F64, radius):
    """||T - T64|| / max(||T64||, ||F64|| * mean radius): the torque error
    measured against the larger of the torque itself and the torque scale of
    the forces (force times lever arm), so that torques that vanish to
    rounding (a sphere pressed straight onto a plane) are not divided by
    their own rounding noise."""
    scale = max(np.linalg.norm(T64), np.linalg.norm(F64) * float(np.mean(radius)))
    d = np.linalg.norm(np.asarray(T) - np.asarray(T64))
    return d / scale if scale > 0 else d


def oracle_coupled(scene):
    """(OracleSPH, OracleDEM) of a CoupledScene with its balls coupled."""
    f = oracle_sph(scene.sph)
    d = oracle_dem(scene.dem)
    sp = scene.sph
    f.couple_balls(d, scene.balls, scene.marker_spacing, scene.marker_h, sp.sound_speed, sp.viscosity, sp.density)
    return f, d


def coupled_momentum(scene, fluid_vel, ball_vel):
    """Total linear momentum of the fluid (mass rho0 dx^3 each) and the balls."""
    sp, dm = scene.sph, scene.dem
    mf = sp.density * sp.spacing ** 3
    mb = dm.density * (4.0 / 3.0) * np.pi * dm.radius ** 3
    return mf * np.asarray(fluid_vel).sum(axis=0) + (mb[:, None] * np.asarray(ball_vel)).sum(axis=0)
