"""Scene descriptions: the reference's example scenes and seeded synthetic
workloads with the sizes of the benchmark configurations.

A scene is plain data (numpy arrays + parameters); ``build_dem`` /
``build_sph`` load it into the solvers.  Generators take explicit seeds.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


def uniform_point_cloud(mn, mx, dx):
    """Inclusive-endpoint lattice of generateUniformPointCloud
    (DEMSPH/pointCloudGeneration.h:7-58): floor(L/dx + 1e-12) + 1 points per
    axis from the low corner, x fastest, then y, then z."""
    eps = 1e-12
    lo = np.minimum(mn, mx).astype(float)
    hi = np.maximum(mn, mx).astype(float)
    n = [max(0, int(math.floor((b - a) / dx + eps)) + 1) for a, b in zip(lo, hi)]
    axes = []
    for k in range(3):
        v = lo[k] + np.arange(n[k]) * dx
        axes.append(v[v <= hi[k] + eps])
    z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)


@dataclass
class HexPBC2D:
    """Periodic cell of a hexagonal x-y packing (DEMSPH/pointCloudGeneration.h:60-80)."""
    min: tuple = (0.0, 0.0, 0.0)
    max: tuple = (0.0, 0.0, 0.0)
    Lx: float = 0.0
    Ly: float = 0.0
    shearX: float = 0.0
    nx: int = 0
    ny: int = 0
    periodicX: bool = False
    periodicY: bool = False


def make_hex_pbc_2d(mn, mx, spacing, periodic_x, periodic_y):
    """makeHexPBC2D (pointCloudGeneration.h:88-140): rows dy = a sqrt(3)/2
    apart; a periodic axis is snapped up to a whole number of steps
    (ceil(L/step - 1e-12)), a bounded one holds floor(L/step + 1e-12) steps."""
    pbc = HexPBC2D(periodicX=bool(periodic_x), periodicY=bool(periodic_y))
    if spacing <= 0.0:
        return pbc
    dx = spacing
    dy = spacing * math.sqrt(3.0) * 0.5
    lx = max(0.0, mx[0] - mn[0])
    ly = max(0.0, mx[1] - mn[1])
    nx = max(1, int(math.ceil(lx / dx - 1e-12))) if periodic_x else max(1, int(math.floor(lx / dx + 1e-12)))
    ny = max(1, int(math.ceil(ly / dy - 1e-12))) if periodic_y else max(1, int(math.floor(ly / dy + 1e-12)))
    pbc.nx, pbc.ny = nx, ny
    pbc.min = tuple(float(v) for v in mn)
    pbc.Lx = nx * dx
    pbc.Ly = ny * dy
    pbc.max = (mn[0] + pbc.Lx if periodic_x else float(mx[0]), mn[1] + pbc.Ly if periodic_y else float(mx[1]),
               float(mx[2]))
    pbc.shearX = 0.5 * dx if (periodic_y and (ny & 1)) else 0.0
    return pbc


def hex_point_cloud(mn, mx, spacing, periodic_x, periodic_y):
    """generateHexPointCloud (pointCloudGeneration.h:152-196): rows along x,
    odd rows shifted by dx/2, z = min z; a bounded axis stops at its max.
    Returns (points, pbc)."""
    pbc = make_hex_pbc_2d(mn, mx, spacing, periodic_x, periodic_y)
    pts = []
    if pbc.nx <= 0 or pbc.ny <= 0 or spacing <= 0.0:
        return np.zeros((0, 3)), pbc
    dx = spacing
    dy = spacing * math.sqrt(3.0) * 0.5
    x0, y0, z0 = pbc.min
    for j in range(pbc.ny):
        y = y0 + j * dy
        if not periodic_y and y >= mx[1]:
            break
        shift = 0.5 * dx if (j & 1) else 0.0
        for i in range(pbc.nx):
            x = x0 + i * dx + shift
            if not periodic_x and x >= mx[0]:
                break
            pts.append((x, y, z0))
    return np.array(pts, float).reshape(-1, 3), pbc


def _normalize(v):
    l2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2]
    if l2 < 1.0e-20:
        return (0.0, 0.0, 0.0)
    inv = 1.0 / math.sqrt(l2)
    return (v[0] * inv, v[1] * inv, v[2] * inv)


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def cylinder_mesh(center, axis, radius, height, n_around, n_height, caps=True):
    """makeCylinderMesh (pointCloudGeneration.h:225-327): nHeight + 1 rings of
    nAround vertices from -h/2 to +h/2 along the axis, two triangles per side
    quad, and (with caps) a centre vertex and a fan per end.  The arithmetic
    follows the reference's order so the vertices come out bit for bit."""
    assert n_around >= 3 and n_height >= 1 and radius > 0 and height > 0
    w = _normalize(axis)
    tmp = (0.0, 0.0, 1.0) if abs(w[2]) < 0.9 else (0.0, 1.0, 0.0)
    u = _normalize(_cross(tmp, w))
    v = _normalize(_cross(w, u))
    verts = []
    for iz in range(n_height + 1):
        t = iz / n_height
        z = (t - 0.5) * height
        c = (center[0] + z * w[0], center[1] + z * w[1], center[2] + z * w[2])
        for ia in range(n_around):
            ang = (2.0 * math.pi) * (ia / n_around)
            ca, sa = math.cos(ang), math.sin(ang)
            verts.append(tuple(c[k] + radius * (ca * u[k] + sa * v[k]) for k in range(3)))

    def vid(iz, ia):
        return iz * n_around + ia % n_around

    t0, t1, t2 = [], [], []
    for iz in range(n_height):
        for ia in range(n_around):
            i00, i01, i10, i11 = vid(iz, ia), vid(iz, ia + 1), vid(iz + 1, ia), vid(iz + 1, ia + 1)
            t0 += [i00, i00]
            t1 += [i10, i11]
            t2 += [i11, i01]
    if caps:
        bottom = len(verts)
        verts.append(tuple(center[k] + (-0.5 * height) * w[k] for k in range(3)))
        top = len(verts)
        verts.append(tuple(center[k] + (0.5 * height) * w[k] for k in range(3)))
        for ia in range(n_around):
            t0.append(bottom); t1.append(vid(0, ia + 1)); t2.append(vid(0, ia))
        for ia in range(n_around):
            t0.append(top); t1.append(vid(n_height, ia)); t2.append(vid(n_height, ia + 1))
    return {"vertices": np.array(verts, float), "tri0": np.array(t0, np.int32), "tri1": np.array(t1, np.int32),
            "tri2": np.array(t2, np.int32)}


def static_sphere_water_level(R, rho_ball, rho_water):
    """waterSurfaceHeightForStaticSphere (DEMSPH/iceCylinderInteraction.cpp:5-35):
    the plane height h in [-R, R] at which the submerged volume fraction
    (R + h)^2 (2R - h) / (4 R^3) equals rho_ball / rho_water, by 80 bisections."""
    if not (R > 0.0) or not (rho_water > 0.0) or not (rho_ball >= 0.0):
        return R
    f = rho_ball / rho_water
    if f <= 0.0:
        return -R
    if f >= 1.0:
        return R
    lo, hi = -R, R
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        b = R + mid
        if (b * b) * (2.0 * R - mid) / (4.0 * R * R * R) < f:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


@dataclass
class DEMScene:
    name: str
    position: np.ndarray
    radius: np.ndarray
    density: np.ndarray
    material: np.ndarray
    velocity: np.ndarray = None
    fixed: np.ndarray = None          # bool per ball (addFixedBall)
    hertz: list = field(default_factory=list)    # rows of setHertzianPair args
    linear: list = field(default_factory=list)   # rows of setLinearPair args
    bonded: list = field(default_factory=list)   # rows of setBondedPair args
    walls: list = field(default_factory=list)    # dicts: vertices, tri0, tri1, tri2, position, material
    clumps: list = field(default_factory=list)   # dicts of addClump args
    bond_initial_contacts: bool = False          # the addInitialCondition hook of the bonded scenes
    buoyancy: tuple = None                       # (rho, Cd, g, u, level)
    periodic: tuple = None                       # setPeriodicBoundary(X, Y, Z)
    minb: tuple = (0, 0, 0)
    maxb: tuple = (1, 1, 1)
    gravity: tuple = (0, 0, -9.81)
    dt: float = 1e-5
    steps: int = 1000

    @property
    def num_moving(self):
        nf = 0 if self.fixed is None else int(np.count_nonzero(self.fixed))
        npeb = sum(len(c["radius"]) for c in self.clumps)
        return self.position.shape[0] - nf + npeb


@dataclass
class SPHScene:
    name: str
    fluid: np.ndarray
    dummy: np.ndarray
    spacing: float
    sound_speed: float
    density: float = 1000.0
    viscosity: float = 1e-3
    minb: tuple = (0, 0, 0)
    maxb: tuple = (1, 1, 1)
    gravity: tuple = (0, 0, -9.81)
    dt: float = 1e-4
    steps: int = 1000


# ---------------------------------------------------------------------------
# Reference example scenes
# ---------------------------------------------------------------------------
def elastic_bounce():
    """DEMSPH/elasticBounce.cpp: one sphere (r 0.01, rho 2000) dropped from
    z = 0 onto a 2-triangle wall at z = -1, undamped linear spring with
    contact time 5 ms, dt = t_c / 50."""
    r, tc = 0.01, 0.005
    m = 4.0 / 3.0 * r ** 3 * math.pi * 2000
    verts = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1]], float)
    s = DEMScene(
        name="elastic_bounce",
        position=np.zeros((1, 3)), radius=np.array([r]), density=np.array([2000.0]), material=np.array([0]),
        linear=[(0, 0, 0.5 * m * math.pi ** 2 / tc / tc, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0)],
        walls=[dict(vertices=verts, tri0=[0, 1], tri1=[1, 2], tri2=[3, 3], position=(0, 0, 0), material=0)],
        minb=(-1, -1, -1), maxb=(1, 1, 1), gravity=(0, 0, -9.81), dt=tc / 50, steps=20000)
    return s


def dam_break_reference():
    """DEMSPH/damBreak.cpp: 21 x 41 x 21 fluid lattice at dx = 0.005 in a
    5H x 2H x 3H tank (H = 0.1) with three dummy layers, open top."""
    H, sp = 0.1, 0.005
    n = int(H / sp)
    sp = H / n
    fluid = uniform_point_cloud(np.array([0.0, 0, 0]), np.array([H, 2 * H, H]), sp)
    tw = 3 * sp
    lo = np.array([0.0, 0, 0]) - tw
    hi = np.array([5 * H, 2 * H, 3 * H]) + tw
    d0 = uniform_point_cloud(lo, hi, sp)
    keep = (d0[:, 0] < 0) | (d0[:, 1] < 0) | (d0[:, 2] < 0) | (d0[:, 0] > 5 * H) | (d0[:, 1] > 2 * H)
    c = 20.0 * math.sqrt(9.81 * H)
    dt = 0.25 * 1.3 * sp / (c + 2.0 * math.sqrt(9.81 * H))
    return SPHScene(name="dam_break_reference", fluid=fluid, dummy=d0[keep], spacing=sp, sound_speed=c,
                    minb=tuple(lo), maxb=tuple(hi), dt=dt, steps=670)


# ---------------------------------------------------------------------------
# Benchmark-sized synthetic scenes
# ---------------------------------------------------------------------------
def ice_cylinder_reference():
    """DEMSPH/iceCylinderInteraction.cpp: a hexagonally packed ice sheet of
    r = 0.1 spheres (rho 900, 100 x 116 rows over 20 x 20 m, periodic rows in
    y) moving at -0.4 m/s in x against a fixed cylinder mesh (radius 1,
    height 6, 36 x 36 segments) at (-1.1, 10, 0); linear contact, parallel
    bonds on the initial contacts, buoyancy + drag against a water plane at
    the static flotation height, dt = t_c / 50."""
    tc, r, den = 0.0002, 0.1, 900.0
    m = r * r * r * math.pi * 4.0 / 3.0 * den
    kn = 0.5 * m * math.pi * math.pi / tc / tc
    E = kn * 2.0 * r / (r * r * math.pi)
    pts, pbc = hex_point_cloud((0.0, 0.0, 0.0), (200 * r, 200 * r, 0.0), 2 * r, False, True)
    mesh = cylinder_mesh((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 1.0, 6.0, 36, 36)
    n = pts.shape[0]
    lin = (kn, kn / 2.6, 0.0, 0.0, 0.1, 0.1, 0.0, 0.0, 0.1, 0.0, 0.0)
    level = static_sphere_water_level(r, den, 1000.0)
    sc = DEMScene(
        name="ice_cylinder", position=pts, radius=np.full(n, r), density=np.full(n, den),
        material=np.zeros(n, np.int32), velocity=np.tile([-0.4, 0.0, 0.0], (n, 1)),
        linear=[(0, 0) + lin, (0, 1) + lin], bonded=[(0, 0, 1.0, E, 2.6, 0.5e6, 0.5e6, 0.1)],
        walls=[dict(mesh, position=(-1.1, 100 * r, 0.0), material=1)],
        minb=(-pbc.max[0], pbc.min[1], -3.0), maxb=(pbc.max[0], pbc.max[1], 3.0), gravity=(0.0, 0.0, -9.81),
        dt=tc / 50.0, steps=int(50.0 / (tc / 50.0)) + 2)
    sc.buoyancy = (1000.0, 0.1, (0.0, 0.0, -9.81), (-0.4, 0.0, 0.0), level)
    sc.bond_initial_contacts = True
    return sc


def dem_periodic_box(n_side=10, radius=0.005, density=2500.0, squeeze=0.985, seed=5, periodic=(True, True, False),
                     E=1e8, nu=0.3, restitution=0.8, mu=0.3, speed=0.05, dt=1e-5):
    """A box exactly tiled by an n_side^3 lattice of Hertz-Mindlin spheres
    (pitch 2 r squeeze, so neighbours overlap by 1.5% of a diameter), with
    seeded random velocities: the lattice is continuous across the box faces,
    so the periodic ghost passes (setPeriodicBoundary) find contacts across
    every periodic face."""
    rng = np.random.default_rng(seed)
    pitch = 2.0 * radius * squeeze
    g = (np.arange(n_side) + 0.5) * pitch
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    p = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    n = p.shape[0]
    L = n_side * pitch
    Es, Gs = hertz_params(E, nu)
    sc = DEMScene(name="dem_periodic_box", position=p, radius=np.full(n, radius), density=np.full(n, density),
                  material=np.zeros(n, np.int32), velocity=rng.uniform(-speed, speed, (n, 3)),
                  hertz=[(0, 0, Es, Gs, restitution, 0.0, 0.0, mu, 0.0, 0.0)], minb=(0.0, 0.0, 0.0),
                  maxb=(L, L, L), gravity=(0.0, 0.0, 0.0), dt=dt, steps=100)
    sc.periodic = tuple(bool(v) for v in periodic)
    return sc


def hertz_params(E, nu):
    """Effective moduli for like materials: E* = E / (2 (1 - nu^2)),
    G* = E / (4 (2 - nu)(1 + nu))."""
    return E / (2 * (1 - nu * nu)), E / (4 * (2 - nu) * (1 + nu))


def dem_drop(n_side=16, spacing=0.012, radius=0.005, density=2500.0, jitter=0.0005, seed=1, plane_gap=0.001,
             E=1e8, nu=0.3, restitution=0.8, mu=0.3, dt=1e-5, steps=1000):
    """n_side^3 Hertz-Mindlin spheres on a jittered lattice dropped onto a
    2-triangle plane wall (the plain DEM bounce workload: 4,096 spheres,
    r 5 mm, rho 2500, 12 mm lattice, +-0.5 mm seeded jitter)."""
    rng = np.random.default_rng(seed)
    g = (np.arange(n_side) + 0.5) * spacing
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    p = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    p += rng.uniform(-jitter, jitter, size=p.shape)
    n = p.shape[0]
    Es, Gs = hertz_params(E, nu)
    zmin = p[:, 2].min() - radius - plane_gap
    L = n_side * spacing
    cell = 2 * radius
    lo = np.array([-2 * cell, -2 * cell, zmin - 2 * cell])
    hi = np.array([L + 2 * cell, L + 2 * cell, p[:, 2].max() + radius + 2 * cell])
    verts = np.array([[lo[0], lo[1], zmin], [hi[0], lo[1], zmin], [hi[0], hi[1], zmin], [lo[0], hi[1], zmin]])
    return DEMScene(
        name="dem_drop", position=p, radius=np.full(n, radius), density=np.full(n, density),
        material=np.zeros(n, np.int32),
        hertz=[(0, 0, Es, Gs, restitution, 0.0, 0.0, mu, 0.0, 0.0)],
        walls=[dict(vertices=verts, tri0=[0, 1], tri1=[1, 2], tri2=[3, 3], position=(0, 0, 0), material=0)],
        minb=tuple(lo), maxb=tuple(hi), dt=dt, steps=steps)


def dem_pack(n_side=16, radius=0.005, density=2500.0, overlap=0.02, seed=3, E=1e8, nu=0.3, restitution=0.8,
             mu=0.3, vel=0.05, dt=1e-5):
    """A dense, touching lattice pack with seeded random velocities and
    spins: every ball starts in contact with its face neighbours, so pair
    forces, friction springs and rolling all act from the first step."""
    rng = np.random.default_rng(seed)
    sp = 2 * radius * (1 - overlap)
    g = (np.arange(n_side) + 0.5) * sp
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    p = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    p += rng.uniform(-0.02 * radius, 0.02 * radius, size=p.shape)
    n = p.shape[0]
    Es, Gs = hertz_params(E, nu)
    L = n_side * sp
    cell = 2 * radius
    lo = np.array([-2 * cell] * 3)
    hi = np.array([L + 2 * cell] * 3)
    s = DEMScene(
        name="dem_pack", position=p, radius=np.full(n, radius), density=np.full(n, density),
        material=np.zeros(n, np.int32),
        hertz=[(0, 0, Es, Gs, restitution, 0.2, 0.1, mu, 0.05, 0.05)],
        minb=tuple(lo), maxb=tuple(hi), gravity=(0, 0, -9.81), dt=dt, steps=100)
    s.velocity = rng.normal(0, vel, size=p.shape)
    s.angvel = rng.normal(0, vel / radius, size=p.shape)
    return s


def sph_dam_break(nx=40, ny=40, nz=80, dx=0.01, tank=(1.6, 0.4, 1.0), layers=3, column_height=0.8, steps=2000):
    """WCSPH dam break with nx*ny*nz fluid particles (default 40x40x80 =
    128,000 at dx = 0.01 in a 0.4 x 0.4 x 0.8 column) inside a tank with
    `layers` dummy layers on the floor and side walls (open top, the rule of
    DEMSPH/damBreak.cpp:25-34); h = 1.3 dx, c0 = 10 sqrt(2 g H),
    dt = 0.25 h / (c0 + 2 sqrt(g H))."""
    gx = (np.arange(nx) + 0.5) * dx
    gy = (np.arange(ny) + 0.5) * dx
    gz = (np.arange(nz) + 0.5) * dx
    z, y, x = np.meshgrid(gz, gy, gx, indexing="ij")
    fluid = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    tw = layers * dx
    lo = np.array([0.0, 0, 0]) - tw
    hi = np.array(tank, float) + tw
    ax = [np.arange(-layers, int(round(t / dx)) + layers) * dx + 0.5 * dx for t in tank]
    zz, yy, xx = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    d0 = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)
    keep = (d0[:, 0] < 0) | (d0[:, 1] < 0) | (d0[:, 2] < 0) | (d0[:, 0] > tank[0]) | (d0[:, 1] > tank[1])
    g = 9.81
    c0 = 10.0 * math.sqrt(2 * g * column_height)
    h = 1.3 * dx
    dt = 0.25 * h / (c0 + 2.0 * math.sqrt(g * column_height))
    return SPHScene(name="sph_dam_break", fluid=fluid, dummy=d0[keep], spacing=dx, sound_speed=c0,
                    minb=tuple(lo), maxb=tuple(hi), dt=dt, steps=steps)


def dem_drop_poly(n, seed, sigma=0.2, ratio=3.0, r0=0.005, density=2500.0, E=1e8, nu=0.3, restitution=0.8,
                  mu=0.3, dt=1e-5):
    """About n Hertz-Mindlin spheres with log-normal radii (sigma, max/min <=
    ratio) on a jittered lattice dropped onto a 2-triangle plane: the DEM drop
    of the scene stream."""
    rng = np.random.default_rng(seed)
    side = max(2, int(round(n ** (1.0 / 3.0))))
    rmax = r0 * math.sqrt(ratio)
    rad = np.exp(np.log(r0) + sigma * rng.standard_normal(side ** 3)).clip(r0 / math.sqrt(ratio), rmax)
    sp = 2.4 * rmax
    g = (np.arange(side) + 0.5) * sp
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    p = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    p += rng.uniform(-0.1 * rmax, 0.1 * rmax, size=p.shape)
    Es, Gs = hertz_params(E, nu)
    zmin = (p[:, 2] - rad).min() - 0.1 * rmax
    L = side * sp
    cell = 2 * rmax
    lo = np.array([-2 * cell, -2 * cell, zmin - 2 * cell])
    hi = np.array([L + 2 * cell, L + 2 * cell, (p[:, 2] + rad).max() + 2 * cell])
    verts = np.array([[lo[0], lo[1], zmin], [hi[0], lo[1], zmin], [hi[0], hi[1], zmin], [lo[0], hi[1], zmin]])
    k = p.shape[0]
    return DEMScene(name="dem_drop_poly", position=p, radius=rad, density=np.full(k, density),
                    material=np.zeros(k, np.int32), hertz=[(0, 0, Es, Gs, restitution, 0.0, 0.0, mu, 0.0, 0.0)],
                    walls=[dict(vertices=verts, tri0=[0, 1], tri1=[1, 2], tri2=[3, 3], position=(0, 0, 0),
                                material=0)],
                    minb=tuple(lo), maxb=tuple(hi), dt=dt)


def dem_agglomerate_drop(n, seed, r=0.005, density=2500.0, E=1e8, nu=0.3, restitution=0.8, mu=0.3, dt=1e-5,
                         bond_E=1.0e7, strength=1.0e6, gap=-0.002):
    """About n spheres of radius r dropped onto a 2-triangle plane, half in
    bonded agglomerates (3 x 3 x 3 cubes of pitch 2r (1 + gap); the default
    gap is a 0.2% overlap, so every face neighbour is a contact of definite
    sign -- none starts at an overlap of rounding size -- and lies in an
    adjacent cell of the 2 r_max grid, whatever the grid's alignment; parallel
    bonds on these initial contacts, normal stiffness bond_E / 2r per unit area,
    k_n / k_s = 2.5, breakable at `strength`), half in rigid 3-sphere clumps
    (collinear pebbles 1.5 r apart, seeded orientations); agglomerates and
    clumps alternate on a lattice of pitch 8r with seeded jitter.  Hertz-
    Mindlin contact, the time step and gravity of dem_drop_poly, so both share
    a DEM batch."""
    rng = np.random.default_rng(seed)
    cells = max(2, int(round(n / 15.0)))
    side = max(2, int(math.ceil(cells ** (1.0 / 3.0))))
    pitch = 8.0 * r
    Es, Gs = hertz_params(E, nu)
    pos = []
    clumps = []
    m_peb = 4.0 / 3.0 * math.pi * r ** 3 * density
    m = 3.0 * m_peb
    I0 = 0.4 * m_peb * r * r
    cube = (np.stack(np.meshgrid(*([np.arange(3.0) - 1.0] * 3), indexing="ij"), -1).reshape(-1, 3)) * 2.0 * r * (1 + gap)
    for k in range(cells):
        i, j, l = k % side, (k // side) % side, k // (side * side)
        c = np.array([(i + 0.5) * pitch, (j + 0.5) * pitch, 2.0 * r + (l + 0.5) * pitch])
        c += rng.uniform(-0.25 * r, 0.25 * r, 3)
        if k % 2 == 0:
            pos.append(c + cube)
        else:
            ax = rng.normal(size=3)
            ax /= np.linalg.norm(ax)
            pts = c + np.outer([-1.0, 0.0, 1.0], ax) * 1.5 * r
            off = 2.0 * m_peb * (1.5 * r) ** 2
            Iax, Iperp = 3 * I0, 3 * I0 + off
            If = Iperp * np.eye(3) + (Iax - Iperp) * np.outer(ax, ax)
            clumps.append(dict(point=pts, radius=[r, r, r], centroid=c, velocity=(0.0, 0.0, 0.0),
                               angularVelocity=(0.0, 0.0, 0.0), mass=m,
                               inertia=(If[0, 0], If[1, 1], If[2, 2], If[0, 1], If[0, 2], If[1, 2]), material=0))
    p = np.concatenate(pos, axis=0)
    nb = p.shape[0]
    L = side * pitch
    lo = np.array([-2 * pitch, -2 * pitch, -2 * r])
    hi = np.array([L + 2 * pitch, L + 2 * pitch, 2.0 * r + (cells // (side * side) + 1) * pitch + pitch])
    verts = np.array([[lo[0], lo[1], 0.0], [hi[0], lo[1], 0.0], [hi[0], hi[1], 0.0], [lo[0], hi[1], 0.0]])
    sc = DEMScene(name="dem_agglomerate_drop", position=p, radius=np.full(nb, r), density=np.full(nb, density),
                  material=np.zeros(nb, np.int32), hertz=[(0, 0, Es, Gs, restitution, 0.0, 0.0, mu, 0.0, 0.0)],
                  bonded=[(0, 0, 1.0, bond_E, 2.5, strength, strength, 0.0)], clumps=clumps,
                  walls=[dict(vertices=verts, tri0=[0, 1], tri1=[1, 2], tri2=[3, 3], position=(0, 0, 0),
                              material=0)],
                  minb=tuple(lo), maxb=tuple(hi), dt=dt)
    sc.bond_initial_contacts = True
    return sc


def bonded_beam_clumps(nx=400, ny=20, nz=20, r=0.001, n_clumps=20_000, seed=11, density=7800.0, E=2.0e11,
                       nu=0.3, restitution=0.5, mu=0.3, tip_load=0.05, dt=1.0e-7, steps=1000):
    """The bonded cantilever beam plus clumps of the DEM stress test: nx x ny x nz
    spheres of radius r on a cubic lattice of pitch 2r (the beam along x),
    parallel bonds on the initial face contacts (normal stiffness 1e12 Pa/m
    and shear stiffness 4e11 Pa/m, i.e. E_b = 1e12 x 2r and k_n/k_s = 2.5; normal
    and shear strengths 5e6 Pa, breakable, gamma = 1, no friction term), the
    x = 0 layer clamped (fixed balls), a seeded random constant load on the tip
    layer; beside the beam n_clumps rigid 3-sphere clumps (collinear pebbles of
    radius r at 1.5 r spacing, seeded orientations) over a 2-triangle floor,
    falling under gravity.  Hertz-Mindlin contact (E, nu, restitution, mu)."""
    rng = np.random.default_rng(seed)
    gx = (np.arange(nx) + 0.5) * 2 * r
    gy = (np.arange(ny) + 0.5) * 2 * r
    gz = (np.arange(nz) + 0.5) * 2 * r + 0.02
    x, y, z = np.meshgrid(gx, gy, gz, indexing="ij")
    beam = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)  # x-major: the first ny*nz are the x = 0 layer
    nb = beam.shape[0]
    fixed = np.zeros(nb, bool)
    fixed[: ny * nz] = True
    Es, Gs = hertz_params(E, nu)
    # clumps on a lattice beside the beam (y > beam), each inside a 6r cube
    side = int(math.ceil(n_clumps ** (1.0 / 3.0)))
    pitch = 6.0 * r
    clumps = []
    y0 = ny * 2 * r + 4 * r
    m = 3.0 * 4.0 / 3.0 * math.pi * r ** 3 * density
    I0 = 0.4 * (m / 3.0) * r * r
    for k in range(n_clumps):
        i, j, l = k % side, (k // side) % side, k // (side * side)
        c = np.array([(i + 0.5) * pitch, y0 + (j + 0.5) * pitch, 0.004 + (l + 0.5) * pitch])
        ax = rng.normal(size=3)
        ax /= np.linalg.norm(ax)
        pts = c + np.outer([-1.0, 0.0, 1.0], ax) * 1.5 * r
        # inertia of three spheres about the centroid: 3 x sphere + 2 x (m/3)(1.5r)^2 off the axis
        off = 2.0 * (m / 3.0) * (1.5 * r) ** 2
        Iax = 3 * I0
        Iperp = 3 * I0 + off
        Ifull = Iperp * np.eye(3) + (Iax - Iperp) * np.outer(ax, ax)
        clumps.append(dict(point=pts, radius=[r, r, r], centroid=c, velocity=(0.0, 0.0, 0.0),
                           angularVelocity=(0.0, 0.0, 0.0), mass=m,
                           inertia=(Ifull[0, 0], Ifull[1, 1], Ifull[2, 2], Ifull[0, 1], Ifull[0, 2], Ifull[1, 2]),
                           material=0))
    L = max(nx * 2 * r, side * pitch)
    lo = np.array([-4 * r, -4 * r, 0.0])
    hi = np.array([L + 4 * r, y0 + side * pitch + 4 * r, max(0.02 + nz * 2 * r, 0.004 + side * pitch) + 8 * r])
    verts = np.array([[lo[0], lo[1], 0.002], [hi[0], lo[1], 0.002], [hi[0], hi[1], 0.002], [lo[0], hi[1], 0.002]])
    sc = DEMScene(name="bonded_beam_clumps", position=beam, radius=np.full(nb, r), density=np.full(nb, density),
                  material=np.zeros(nb, np.int32), fixed=fixed,
                  hertz=[(0, 0, Es, Gs, restitution, 0.0, 0.0, mu, 0.0, 0.0)],
                  bonded=[(0, 0, 1.0, 1.0e12 * 2 * r, 2.5, 5.0e6, 5.0e6, 0.0)],
                  clumps=clumps,
                  walls=[dict(vertices=verts, tri0=[0, 1], tri1=[1, 2], tri2=[3, 3], position=(0, 0, 0),
                              material=0)],
                  minb=tuple(lo), maxb=tuple(hi), dt=dt, steps=steps)
    sc.bond_initial_contacts = True
    load = np.zeros((nb, 3))
    tip = np.arange(nb - ny * nz, nb)
    d = rng.normal(size=(tip.size, 3))
    load[tip] = tip_load * d / np.linalg.norm(d, axis=1, keepdims=True)
    sc.constant_force = load
    return sc


def ice_sheet_on_water(n_side=930, r=0.002, jitter=0.05, dx=0.004, water_layers=2, fluid=2_000_000, layers=3, seed=13,
                       density=917.0, E=9.0e9, nu=0.3, speed=0.5, cyl_segments=(100, 100), dem_dt=2.0e-7,
                       dem_substeps=1, steps=100):
    """The coupled ice-cylinder stress scene: a hexagonally packed sheet of about
    n_side^2 bonded spheres (radius r with seeded +-jitter, density 917,
    Hertz-Mindlin with E = 9e9) moving at `speed` in -x towards a fixed
    cylinder mesh (n_around x n_height segments: 20,000 triangles by
    default), floating on a WCSPH water layer of `water_layers` lattice layers
    at spacing dx under the sheet and ahead of it, about `fluid` particles,
    over `layers` dummy layers of floor; the sheet's balls are coupled
    to the water particle by particle (one marker each when r <= 3 dx / 4).
    The fluid step is dem_dt x dem_substeps (far below its own CFL limit; the
    bond stiffness sets the step).  Returns a CoupledScene."""
    rng = np.random.default_rng(seed)
    pitch = 2 * r
    rows = int(round(n_side / (math.sqrt(3) / 2)))
    cols = n_side
    W, H = cols * pitch, rows * pitch * math.sqrt(3) / 2
    j = np.arange(rows)
    i = np.arange(cols)
    ii, jj = np.meshgrid(i, j, indexing="xy")
    px = (ii + 0.5 + 0.5 * (jj % 2)) * pitch
    py = (jj + 0.5) * pitch * math.sqrt(3) / 2
    zw = water_layers * dx  # water surface
    pz = np.full(px.shape, zw)  # centres at the surface: half submerged
    pos = np.stack([px.ravel(), py.ravel(), pz.ravel()], axis=1)
    n = pos.shape[0]
    rad = r * (1.0 + rng.uniform(-jitter, jitter, n))
    # the water: a lattice under the sheet, extended ahead of it (-x) to about `fluid` particles
    nyw = int(H / dx)
    nxw = max(int(W / dx), int(round(fluid / (water_layers * nyw))))
    margin = nxw * dx - W
    Ly = H
    gx = (np.arange(nxw) + 0.5) * dx - margin
    gy = (np.arange(nyw) + 0.5) * dx
    gz = (np.arange(water_layers) + 0.5) * dx
    zz, yy, xx = np.meshgrid(gz, gy, gx, indexing="ij")
    fluid = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)
    tw = layers * dx
    lo = np.array([-margin, 0.0, 0.0]) - tw
    hi = np.array([W, Ly, zw + 8 * r + 4 * dx]) + tw
    ax = [np.arange(int(round((h0 - l0) / dx))) * dx + l0 + 0.5 * dx for l0, h0 in zip(lo, hi)]
    dz = ax[2][ax[2] < 0]
    zz, yy, xx = np.meshgrid(dz, ax[1], ax[0], indexing="ij")
    floor = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)
    g = 9.81
    c0 = 10.0 * math.sqrt(2 * g * zw)
    h = 1.3 * dx
    sph = SPHScene(name="ice_sheet_water", fluid=fluid, dummy=floor, spacing=dx, sound_speed=c0, density=1000.0,
                   minb=tuple(lo), maxb=tuple(hi), gravity=(0.0, 0.0, -g), dt=dem_dt * dem_substeps, steps=steps)
    Es, Gs = hertz_params(E, nu)
    n_around, n_height = cyl_segments
    cyl_r = 0.05 * H  # ahead of the sheet's leading (-x) edge
    mesh = cylinder_mesh((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), cyl_r, 0.1, n_around, n_height, caps=False)
    dem = DEMScene(name="ice_sheet", position=pos, radius=rad, density=np.full(n, density),
                   material=np.zeros(n, np.int32), velocity=np.tile([-speed, 0.0, 0.0], (n, 1)),
                   hertz=[(0, 0, Es, Gs, 0.3, 0.0, 0.0, 0.2, 0.0, 0.0), (0, 1, Es, Gs, 0.3, 0.0, 0.0, 0.2, 0.0, 0.0)],
                   bonded=[(0, 0, 1.0, E, 2.6, 0.5e6, 0.5e6, 0.1)],
                   walls=[dict(mesh, position=(-(cyl_r + 4 * r), 0.5 * H, zw - 0.05), material=1)],
                   minb=tuple(lo), maxb=tuple(hi), gravity=(0.0, 0.0, -g), dt=dem_dt, steps=steps)
    dem.bond_initial_contacts = True
    return CoupledScene(name="ice_sheet_on_water", sph=sph, dem=dem, balls=np.arange(n, dtype=np.int32),
                        marker_spacing=dx, marker_h=h, dem_substeps=dem_substeps, steps=steps)


def sph_column(n, sound_speed, dt, dx=0.01, layers=3):
    """A dam break with about n fluid particles: a nx x nx x 2nx column at the
    left end of a tank four columns long and 1.25 columns high, three dummy
    layers, open top (the dam break of the scene stream).  Sound speed and dt
    are given so that scenes of one stream share them."""
    nx = max(2, int(round((n / 2.0) ** (1.0 / 3.0))))
    nz = 2 * nx
    tank = (4 * nx * dx, nx * dx, 1.25 * nz * dx)
    gx = (np.arange(nx) + 0.5) * dx
    gz = (np.arange(nz) + 0.5) * dx
    z, y, x = np.meshgrid(gz, gx, gx, indexing="ij")
    fluid = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    tw = layers * dx
    lo = np.array([0.0, 0, 0]) - tw
    hi = np.array(tank, float) + tw
    ax = [np.arange(-layers, int(round(t / dx)) + layers) * dx + 0.5 * dx for t in tank]
    zz, yy, xx = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    d0 = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)
    keep = (d0[:, 0] < 0) | (d0[:, 1] < 0) | (d0[:, 2] < 0) | (d0[:, 0] > tank[0]) | (d0[:, 1] > tank[1])
    return SPHScene(name="sph_column", fluid=fluid, dummy=d0[keep], spacing=dx, sound_speed=sound_speed,
                    minb=tuple(lo), maxb=tuple(hi), dt=dt)


@dataclass
class CoupledScene:
    """A fluid scene, a DEM scene and the balls coupled particle by particle."""
    name: str
    sph: SPHScene
    dem: DEMScene
    balls: np.ndarray            # DEM indices of the coupled balls
    marker_spacing: float
    marker_h: float
    dem_substeps: int = 1
    steps: int = 100


def balls_in_tank(nx=24, ny=24, depth=24, dx=0.01, layers=3, balls=((0.5, 0.5, 0.5, 4.0, 500.0),),
                  ball_velocity=None, headroom=12, dem_substeps=2, gravity=(0.0, 0.0, -9.81), walls=True,
                  E=1e7, nu=0.3, restitution=0.5, mu=0.3, steps=100):
    """DEM balls immersed in a tank of still water: an nx x ny x depth
    lattice of fluid (spacing dx) in a tank with `layers` dummy layers on the
    floor and the four sides (open top, `headroom` cells above the water), and
    balls given as (x, y, z as fractions of the water block, radius in dx,
    density).  Fluid particles closer than radius + dx/2 to a ball centre are
    removed.  The DEM scene has the balls over a 2-triangle floor plane at
    the tank floor (Hertz-Mindlin, E, nu, restitution, mu); its time step is
    the fluid's divided by dem_substeps.  Fluid h = 1.3 dx, c0 = 10 sqrt(2 g H),
    dt = 0.25 h / (c0 + 2 sqrt(g H)); markers use dx and h.  walls=False
    drops the dummies and the floor (a free block, for momentum checks)."""
    H = depth * dx
    g = max(9.81, abs(gravity[2]))
    c0 = 10.0 * math.sqrt(2 * g * H)
    h = 1.3 * dx
    dt = 0.25 * h / (c0 + 2.0 * math.sqrt(g * H))
    gx = (np.arange(nx) + 0.5) * dx
    gy = (np.arange(ny) + 0.5) * dx
    gz = (np.arange(depth) + 0.5) * dx
    z, y, x = np.meshgrid(gz, gy, gx, indexing="ij")
    fluid = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    block = np.array([nx * dx, ny * dx, H])
    bpos = np.array([[b[0] * block[0], b[1] * block[1], b[2] * block[2]] for b in balls], float)
    brad = np.array([b[3] * dx for b in balls], float)
    bden = np.array([b[4] for b in balls], float)
    keep = np.ones(len(fluid), bool)
    for c, r in zip(bpos, brad):
        keep &= np.linalg.norm(fluid - c, axis=1) >= r + 0.5 * dx
    fluid = fluid[keep]
    tank = (nx * dx, ny * dx, (depth + headroom) * dx)
    tw = layers * dx
    lo = np.array([0.0, 0, 0]) - tw
    hi = np.array(tank, float) + tw
    if walls:
        ax = [np.arange(-layers, int(round(t / dx)) + layers) * dx + 0.5 * dx for t in tank]
        zz, yy, xx = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
        d0 = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)
        side = ((d0[:, 0] < 0) | (d0[:, 1] < 0) | (d0[:, 2] < 0) | (d0[:, 0] > tank[0]) | (d0[:, 1] > tank[1]))
        dummy = d0[side]
    else:
        dummy = np.zeros((0, 3))
    sph = SPHScene(name="balls_in_tank_fluid", fluid=fluid, dummy=dummy, spacing=dx, sound_speed=c0,
                   minb=tuple(lo), maxb=tuple(hi), gravity=tuple(gravity), dt=dt, steps=steps)
    Es, Gs = hertz_params(E, nu)
    k = len(bpos)
    wl = []
    if walls:
        verts = np.array([[lo[0], lo[1], 0.0], [hi[0], lo[1], 0.0], [hi[0], hi[1], 0.0], [lo[0], hi[1], 0.0]])
        wl = [dict(vertices=verts, tri0=[0, 1], tri1=[1, 2], tri2=[3, 3], position=(0, 0, 0), material=0)]
    vel = None if ball_velocity is None else np.asarray(ball_velocity, float).reshape(k, 3)
    dem = DEMScene(name="balls_in_tank_balls", position=bpos, radius=brad, density=bden,
                   material=np.zeros(k, np.int32), velocity=vel,
                   hertz=[(0, 0, Es, Gs, restitution, 0.0, 0.0, mu, 0.0, 0.0)], walls=wl,
                   minb=tuple(lo), maxb=tuple(hi), gravity=tuple(gravity), dt=dt / dem_substeps, steps=steps)
    return CoupledScene(name="balls_in_tank", sph=sph, dem=dem, balls=np.arange(k, dtype=np.int32),
                        marker_spacing=dx, marker_h=h, dem_substeps=dem_substeps, steps=steps)


# ---------------------------------------------------------------------------
# Loading into the solvers
# ---------------------------------------------------------------------------
def build_dem(scene: DEMScene, precision="mixed", stream=None, initialize=True, configure=None):
    """A DEMSolver loaded with the scene (and initialised); `configure(solver)`
    runs before initialisation (cell size, capacities)."""
    from .solvers import DEMSolver

    s = DEMSolver(stream)
    for row in scene.hertz:
        s.setHertzianPair(*row)
    for row in scene.linear:
        s.setLinearPair(*row)
    for row in scene.bonded:
        s.setBondedPair(*row)
    fixed = np.zeros(scene.position.shape[0], bool) if scene.fixed is None else scene.fixed
    # keep the caller's ball order: add runs of moving / fixed balls in sequence
    idx = np.arange(scene.position.shape[0])
    starts = np.flatnonzero(np.diff(np.r_[-1, fixed.astype(int)]) != 0)
    bounds = list(starts) + [len(idx)]
    for a, b in zip(bounds[:-1], bounds[1:]):
        sl = slice(a, b)
        if fixed[a]:
            s.addFixedBalls(scene.position[sl], scene.radius[sl], scene.material[sl])
        else:
            vel = None if scene.velocity is None else scene.velocity[sl]
            w = getattr(scene, "angvel", None)
            s.addBalls(scene.position[sl], vel, None if w is None else w[sl], scene.radius[sl], scene.density[sl],
                       scene.material[sl])
    for c in scene.clumps:
        s.addClump(c["point"], c["radius"], c["centroid"], c["velocity"], c["angularVelocity"], c["mass"],
                   c["inertia"], c["material"])
    for k, w in enumerate(scene.walls):
        s.addMeshWall(w["vertices"], w["tri0"], w["tri1"], w["tri2"], w["position"], materialID=w["material"])
        if "velocity" in w:
            s.setMeshWallMotion(k, w["velocity"], w.get("angularVelocity", (0, 0, 0)))
    if scene.buoyancy is not None:
        s.setBuoyancyDrag(*scene.buoyancy)
    if getattr(scene, "constant_force", None) is not None:
        s.setConstantForce(scene.constant_force)
    if scene.periodic is not None:
        s.setPeriodicBoundary(*scene.periodic)
    if configure is not None:
        configure(s)
    if initialize:
        s.initialize(scene.minb, scene.maxb, scene.gravity, scene.dt, precision)
        if scene.bond_initial_contacts:
            p = s.getPairs(0)
            s.addBondedInteraction(p["objectPointed"], p["objectPointing"], scene.position)
    return s


def build_sph(scene: SPHScene, precision="fp64", stream=None, initialize=True, configure=None):
    """A WCSPHSolver loaded with the scene (and initialised); `configure(solver)`
    runs before initialisation (cell size, skin, list headroom)."""
    from .solvers import WCSPHSolver

    s = WCSPHSolver(stream)
    s.addSPHs(scene.fluid, None, scene.sound_speed, scene.spacing, scene.density, scene.viscosity)
    s.addDummies(scene.dummy, None, scene.sound_speed, scene.spacing, scene.density, scene.viscosity)
    if configure is not None:
        configure(s)
    if initialize:
        s.initialize(scene.minb, scene.maxb, scene.gravity, scene.dt, precision)
    return s


def build_coupled(scene: CoupledScene, precision="fp64", stream=None):
    """(WCSPHSolver, DEMSolver, DEMSPHCoupling) of a coupled scene, initialised."""
    from .solvers import DEMSPHCoupling

    f = build_sph(scene.sph, precision, stream)
    d = build_dem(scene.dem, precision, stream)
    c = DEMSPHCoupling(f, d)
    sp = scene.sph
    c.addBalls(scene.balls, scene.marker_spacing, scene.marker_h, sp.sound_speed, sp.viscosity, sp.density)
    return f, d, c
