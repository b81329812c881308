"""DEM parity on the GPU: the native library against the FP64 oracle and the
reference's elasticBounce frames.

Tolerances: FP64 mode reproduces the reference arithmetic, so it is held to
1e-10 relative (rounding only).  Mixed mode (FP32 force laws, FP64 state and
springs) is held to the 1e-5 relative force error of the target.
"""
import os

import numpy as np
import pytest

import this_studio_b200 as tsb
from this_studio_b200 import scenes
from this_studio_b200.scenes import build_dem

from .helpers import oracle_dem, pair_keys, rel_err

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = {"fp64": 1e-10, "mixed": 1e-5}


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_elastic_bounce_matches_reference_frames(gpu, prec):
    fx = np.load(os.path.join(GOLDEN, "elastic_bounce.npz"))
    s = build_dem(scenes.elastic_bounce(), prec)
    worst = 0.0
    for f in range(1, 201):
        s.step(100)
        assert s.stepIndex()[0] == fx["step"][f]
        b = s.getBall()
        worst = max(worst, np.abs(b["position"][0] - fx["position"][f]).max(),
                    np.abs(b["velocity"][0] - fx["velocity"][f]).max())
    assert worst < (1e-9 if prec == "fp64" else 2e-5), worst


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_pack_pairs_bit_exact_and_forces(gpu, oracle_lib, prec):
    sc = scenes.dem_pack(n_side=10)
    o = oracle_dem(sc)
    g = build_dem(sc, prec)
    po, pg = o.pairs(0), g.getPairs(0)
    assert len(po["a"]) > 2000
    # same pairs in the same CSR order as the reference's count/write kernels
    np.testing.assert_array_equal(pg["objectPointed"], po["a"])
    np.testing.assert_array_equal(pg["objectPointing"], po["b"])
    # advance both through a rebuild (every 5th step) and compare the state
    o.step(7)
    g.step(7)
    bo, bg = o.balls(), g.getBall()
    assert rel_err(bg["position"] - sc.position, bo["pos"] - sc.position) < 100 * TOL[prec]
    po, pg = o.pairs(0), g.getPairs(0)
    assert np.array_equal(np.sort(pair_keys(pg["objectPointed"], pg["objectPointing"])),
                          np.sort(pair_keys(po["a"], po["b"])))
    # per-step forces from identical states: load the oracle state into the GPU
    g.setBall(bo["pos"], bo["vel"], bo["angvel"])
    o.neighbor_search()
    g.neighborSearch()
    po = o.pairs(0)
    g.importSprings(po["a"], po["b"], po["sliding"], po["rolling"], po["torsion"])
    pg = g.getPairs(0)
    np.testing.assert_array_equal(pg["objectPointed"], po["a"])
    np.testing.assert_array_equal(pg["objectPointing"], po["b"])
    hdt = 0.5 * sc.dt
    o.eval_forces(hdt)
    g.evalForces(hdt)
    fo, fg = o.balls(), g.getBall()
    ef, et = rel_err(fg["force"], fo["force"]), rel_err(fg["torque"], fo["torque"])
    print(f"{prec}: force rel err {ef:.3e} torque rel err {et:.3e}")
    assert ef < TOL[prec] and et < TOL[prec]
    po, pg = o.pairs(0), g.getPairs(0)
    assert rel_err(pg["sliding"], po["sliding"]) < TOL[prec]
    assert rel_err(pg["rolling"], po["rolling"]) < 10 * TOL[prec]
    # internal forces balance
    f = fg["force"]
    assert np.abs(f.sum(0)).max() < (1e-12 if prec == "fp64" else 1e-6) * np.abs(f).sum()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_drop_onto_plane_trajectory(gpu, oracle_lib, prec):
    sc = scenes.dem_drop(n_side=8, plane_gap=0.0)
    sc.steps = 300
    o = oracle_dem(sc)
    g = build_dem(sc, prec)
    o.step(sc.steps)
    g.step(sc.steps)
    bo, bg = o.balls(), g.getBall()
    e = rel_err(bg["velocity"], bo["vel"])
    print(f"{prec}: velocity rel err after {sc.steps} steps {e:.3e}")
    assert e < 1e3 * TOL[prec]
    wo, wg = o.pairs(1), g.getPairs(1)
    assert np.array_equal(np.sort(pair_keys(wg["objectPointed"], wg["objectPointing"])),
                          np.sort(pair_keys(wo["a"], wo["b"])))


def _beam():
    """DEMSPH/bondedParticleBeam.cpp at reduced length: a fixed ball and 10
    balls in a row, bonds from the initial contacts, a ramped tip load and
    global damping."""
    n, L = 10, 4.0
    r = L / n / 2.0
    p = np.array([[(i) * 2 * r, 0, 0] for i in range(n + 1)], float)
    fixed = np.zeros(n + 1, bool)
    fixed[0] = True
    sc = scenes.DEMScene(name="beam", position=p, radius=np.full(n + 1, r), density=np.full(n + 1, 7800.0),
                         material=np.zeros(n + 1, np.int32), fixed=fixed,
                         bonded=[(0, 0, 1.0, 200e9, 2.6, 0.0, 0.0, 0.0)], bond_initial_contacts=True,
                         minb=(0, -r, -r), maxb=(L, r, r), gravity=(0, 0, 0), dt=1e-5)
    f = np.zeros((n + 1, 3))
    f[n] = (0, 0, 100e3)
    return sc, f


def test_bonded_beam(gpu, oracle_lib):
    sc, f = _beam()
    o = oracle_dem(sc)
    o.set_constant_force(f, ramp=1.0)
    o.set_global_damping(0.1)
    g = build_dem(sc, "fp64")
    g.setConstantForce(f, rampTime=1.0)
    g.setGlobalDamping(0.1)
    assert o.bonds()["a"].shape[0] == 10
    o.step(3000)
    g.step(3000)
    bo, bg = o.bonds(), g.getBondedInteraction()
    np.testing.assert_array_equal(bg["isBonded"], bo["ok"])
    assert rel_err(bg["normalForce"], bo["normal_force"]) < 1e-8
    assert rel_err(bg["shearForce"], bo["shear_force"]) < 1e-8
    assert rel_err(g.getBall()["position"], o.balls()["pos"]) < 1e-10


def test_clumps_fall_onto_plane(gpu, oracle_lib):
    rng = np.random.default_rng(5)
    r = 0.004
    sc = scenes.dem_drop(n_side=4, plane_gap=0.0005)
    sc.position = sc.position[:1]
    sc.radius, sc.density, sc.material = sc.radius[:1], sc.density[:1], sc.material[:1]
    for k in range(12):
        c = np.array([0.01 + 0.012 * (k % 4), 0.01 + 0.012 * (k // 4), 0.012])
        ax = rng.normal(size=3)
        ax /= np.linalg.norm(ax)
        pts = c + np.outer([-1, 0, 1], ax) * 1.5 * r
        m = 3 * 4 / 3 * np.pi * r ** 3 * 2500
        I = 0.4 * m * r * r + m * 1.5 * r * 1.5 * r * 2 / 3
        sc.clumps.append(dict(point=pts, radius=[r, r, r], centroid=c, velocity=(0, 0, -0.1),
                              angularVelocity=tuple(rng.normal(0, 5, 3)), mass=m,
                              inertia=(I, I, I, 0, 0, 0), material=0))
    sc.steps = 400
    o = oracle_dem(sc)
    g = build_dem(sc, "fp64")
    o.step(sc.steps)
    g.step(sc.steps)
    co, cg = o.clumps(), g.getClump()
    assert rel_err(cg["position"], co["pos"]) < 1e-10
    assert rel_err(cg["orientation"], co["q"]) < 1e-10
    assert rel_err(g.getBall()["velocity"], o.balls()["vel"]) < 1e-8


def test_buoyancy_drag(gpu, oracle_lib):
    sc = scenes.dem_drop(n_side=5, plane_gap=0.002)
    lvl = float(sc.position[:, 2].mean())
    sc.buoyancy = (1000.0, 0.1, (0, 0, -9.81), (-0.4, 0, 0), lvl)
    sc.steps = 200
    o = oracle_dem(sc)
    g = build_dem(sc, "fp64")
    o.step(sc.steps)
    g.step(sc.steps)
    assert rel_err(g.getBall()["velocity"], o.balls()["vel"]) < 1e-9


def test_overflow_regrowth_keeps_results(gpu, oracle_lib):
    """Polydisperse pack where some balls have many more partners than the
    initial list capacity guess; the library regrows and replays."""
    rng = np.random.default_rng(11)
    n = 600
    p = rng.uniform(0, 0.06, size=(n, 3))
    rad = np.exp(rng.normal(np.log(0.003), 0.35, size=n)).clip(0.0015, 0.0045)
    Es, Gs = scenes.hertz_params(1e7, 0.3)
    sc = scenes.DEMScene(name="poly", position=p, radius=rad, density=np.full(n, 2500.0),
                         material=np.zeros(n, np.int32), hertz=[(0, 0, Es, Gs, 0.5, 0, 0, 0.4, 0, 0)],
                         minb=(-0.01, -0.01, -0.01), maxb=(0.07, 0.07, 0.07), dt=2e-6)
    o = oracle_dem(sc)
    g = build_dem(sc, "fp64")
    o.step(20)
    g.step(20)
    po, pg = o.pairs(0), g.getPairs(0)
    assert np.array_equal(pg["objectPointed"], po["a"]) and np.array_equal(pg["objectPointing"], po["b"])
    assert rel_err(g.getBall()["position"], o.balls()["pos"]) < 1e-10


def test_launch_counter_moves(gpu):
    s = build_dem(scenes.dem_drop(n_side=4), "mixed")
    k0 = tsb.kernel_launches()
    s.step(5)
    assert tsb.kernel_launches() > k0


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_wall_contacts_at_the_mesh_box_edge(gpu, oracle_lib, prec):
    """Balls beside the edges and corners of a square plane wall, at
    distances just inside and just outside their radius from it: those
    within reach touch an edge or a vertex, the others are skipped before the
    triangle walk by the mesh-box test.  Pair sets and states against the
    oracle, which walks every triangle."""
    r, L = 0.005, 0.1
    d = np.array([0.5, 0.9, 0.999, 1.001, 1.5]) * r
    corners = np.array([[L, L], [0, 0], [L, 0], [0, L]])
    p = []
    for k, e in enumerate(d):
        y = 0.1 * L + 0.15 * L * k  # 15 mm apart along each edge: no two balls touch
        p += [[L + e, y, 0.0], [-e, y + 0.05 * L, 0.0], [y, L + e, 0.0],  # beside three edges
              [y + 0.02 * L, 0.5 * L, e], [y + 0.02 * L, 0.75 * L, -e]]   # above / below the face
        if k < 4:  # beside a corner, outwards along its diagonal
            c = corners[k]
            out = np.sign(c - 0.5 * L)
            p.append([c[0] + out[0] * e / np.sqrt(2), c[1] + out[1] * e / np.sqrt(2), 0.0])
    p = np.array(p)
    n = len(p)
    rng = np.random.default_rng(2)
    v = rng.uniform(-0.05, 0.05, size=(n, 3))
    Es, Gs = scenes.hertz_params(1e8, 0.3)
    verts = np.array([[0, 0, 0], [L, 0, 0], [L, L, 0], [0, L, 0]], float)
    sc = scenes.DEMScene(name="box_edge", position=p, radius=np.full(n, r), density=np.full(n, 2500.0),
                         material=np.zeros(n, np.int32), velocity=v,
                         hertz=[(0, 0, Es, Gs, 0.8, 0.0, 0.0, 0.3, 0.0, 0.0)],
                         walls=[dict(vertices=verts, tri0=[0, 1], tri1=[1, 2], tri2=[3, 3], position=(0, 0, 0),
                                     material=0)],
                         minb=(-0.02, -0.02, -0.02), maxb=(L + 0.02, L + 0.02, 0.02), gravity=(0.0, 0.0, 0.0),
                         dt=1e-5, steps=20)
    o = oracle_dem(sc)
    g = build_dem(sc, prec)
    for k, steps in enumerate((1, sc.steps - 1)):
        o.step(steps)
        g.step(steps)
        wo, wg = o.pairs(1), g.getPairs(1)
        assert np.array_equal(np.sort(pair_keys(wg["objectPointed"], wg["objectPointing"])),
                              np.sort(pair_keys(wo["a"], wo["b"])))
        if k == 0:  # every ball within reach (18 of them) is a candidate after the first step
            assert len({int(b) for b in wg["objectPointed"]}) >= 15
    bo, bg = o.balls(), g.getBall()
    e = rel_err(bg["velocity"], bo["vel"])
    print(f"{prec}: {len(wg['objectPointed'])} wall pairs after {sc.steps} steps, velocity rel err {e:.2e}")
    assert e < 1e3 * TOL[prec]
