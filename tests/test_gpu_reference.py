"""The reference's own CUDA kernels (built from its sources into
oracle/_ref by oracle/Makefile.ref) against this library, on the same GPU:
pair lists in the same order, forces and short trajectories, and the step
time of both on the benchmark workload."""
import time

import numpy as np
import pytest

from this_studio_b200 import scenes
from this_studio_b200.scenes import build_dem, build_sph

from .helpers import pair_keys, rel_err, torque_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    from oracle import ref_harness

    if not ref_harness.available():
        pytest.skip("oracle/_ref/libdemsph_ref.so not built (make -f oracle/Makefile.ref)")
    return ref_harness


def test_sph_pairs_and_trajectory_match_reference_kernels(gpu, ref):
    import torch

    sc = scenes.dam_break_reference()
    r = ref.RefSPH(sc, torch)
    g = build_sph(sc, "fp64")
    assert rel_err(g.getDummy()["normal"], r.state()["dummy_normal"]) < 1e-13
    a, b = g.getPairs(2)
    ra, rb = r.pairs(2)
    np.testing.assert_array_equal(a, ra)
    np.testing.assert_array_equal(b, rb)
    r.neighbor_search()
    g.neighborSearch()
    for which in (0, 1):
        a, b = g.getPairs(which)
        ra, rb = r.pairs(which)
        np.testing.assert_array_equal(a, ra)
        np.testing.assert_array_equal(b, rb)
    r.step(30)
    g.step(30)
    s, rs = g.getSPH(), r.state()
    e = rel_err(s["position"] - sc.fluid, rs["pos"] - sc.fluid)
    print(f"30 steps vs reference kernels: displacement rel err {e:.2e}")
    assert e < 1e-10
    assert rel_err(s["density"] - 1000.0, rs["rho"] - 1000.0) < 1e-9
    assert rel_err(s["acceleration"], rs["acc"]) < 1e-9


def test_dem_pairs_and_forces_match_reference_kernels(gpu, ref):
    import torch

    sc = scenes.dem_pack(n_side=12)
    r = ref.RefDEMPairs(sc, torch)
    r.neighbor_search()
    g = build_dem(sc, "fp64")
    ra, rb = r.pairs()
    pg = g.getPairs(0)
    assert len(ra) > 3000
    np.testing.assert_array_equal(pg["objectPointed"], ra)
    np.testing.assert_array_equal(pg["objectPointing"], rb)
    fr, tr = r.forces(0.5 * sc.dt)
    g.evalForces(0.5 * sc.dt)
    b = g.getBall()
    ef, et = rel_err(b["force"], fr), rel_err(b["torque"], tr)
    print(f"DEM forces vs reference kernels: force {ef:.2e} torque {et:.2e}")
    assert ef < 1e-12 and et < 1e-12
    g2 = build_dem(sc, "mixed")
    g2.evalForces(0.5 * sc.dt)
    b2 = g2.getBall()
    print(f"mixed precision vs reference kernels: force {rel_err(b2['force'], fr):.2e}")
    assert rel_err(b2["force"], fr) < 1e-5


def test_step_time_against_reference_kernels(gpu, ref):
    """Both on the benchmark workload (128,000 fluid, 150,216 dummies)."""
    import torch

    sc = scenes.sph_dam_break()
    r = ref.RefSPH(sc, torch)
    r.step(3)
    torch.cuda.synchronize()
    n = 20
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    r.step(n)
    e1.record()
    e1.synchronize()
    ref_ms = e0.elapsed_time(e1) / n
    out = {}
    for prec in ("fp64", "mixed"):
        g = build_sph(sc, prec)
        g.step(3)
        torch.cuda.synchronize()
        e0.record()
        g.step(n)
        e1.record()
        e1.synchronize()
        out[prec] = e0.elapsed_time(e1) / n
    nf = sc.fluid.shape[0]
    print(f"reference CUDA build: {ref_ms:.3f} ms/step = {nf / ref_ms * 1e3:.3e} particle-steps/s; "
          f"this library fp64 {out['fp64']:.3f} ms/step ({ref_ms / out['fp64']:.1f}x), "
          f"mixed {out['mixed']:.3f} ms/step ({ref_ms / out['mixed']:.1f}x)")
    assert out["fp64"] < ref_ms


# --------------------------------------------------------------------------
# Bonds, mesh walls and the buoyancy-drag hook against the reference kernels
# (calBondedForceTorqueKernel, contactKernel.cu:535-655; updateBallTriangleContact
# + calBallWallContactForceTorqueKernel, :261-533; addBuoyancyDragKernel,
# externalForceTorque.cu:79-133), replayed by oracle/ref_harness.RefDEM.
#
# Two checks each: a short trajectory in FP64 (both sides integrate the same
# step loop; rounding only), and one force evaluation in both precisions from
# an identical state (the reference's balls, springs and bond state loaded
# into this library), where mixed precision must stay within the 1e-5
# relative force error of the target.
#
# The reference sets each object's interactionStart / End to -1 only when it
# allocates them (interaction.h:73-84), so a ball (or triangle) that loses all
# its incoming pairs at a rebuild keeps a range into the previous list, and
# sumObjectPointingForceTorqueFromInteractionKernel then adds unrelated
# pairs' forces to it (quirk Q7; on the bonded block below 12 of 1,251 bonds
# end differently after 20 steps).  This library rebuilds those ranges from
# scratch; the replay does the same (RefDEM.correct_q7) for these checks.
TOL_STATE = {"fp64": 1e-12, "mixed": 1e-5}


def _bonded_block(nx=24, ny=5, nz=5, r=0.001, pitch=2.19, seed=4):
    """A bonded block (parallel bonds on the initial contacts, x = 0 layer
    fixed) whose balls move with seeded random velocities and spins: bond
    increments from the first step, some bonds breaking, some contact pairs
    dropping out of the list while their bond holds."""
    rng = np.random.default_rng(seed)
    g = lambda k: (np.arange(k) + 0.5) * pitch * r
    x, y, z = np.meshgrid(g(nx), g(ny), g(nz), indexing="ij")
    p = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    p += rng.uniform(-0.01 * r, 0.01 * r, size=p.shape)
    n = p.shape[0]
    fixed = np.zeros(n, bool)
    fixed[: ny * nz] = True
    Es, Gs = scenes.hertz_params(1e9, 0.3)
    sc = scenes.DEMScene(name="bonded_block", position=p, radius=np.full(n, r), density=np.full(n, 2500.0),
                         material=np.zeros(n, np.int32), fixed=fixed,
                         hertz=[(0, 0, Es, Gs, 0.5, 0.2, 0.1, 0.3, 0.05, 0.05)],
                         bonded=[(0, 0, 1.0, 2.0e9, 2.5, 5.0e6, 5.0e6, 0.3)], bond_initial_contacts=True,
                         minb=(-4 * r, -4 * r, -4 * r), maxb=(nx * pitch * r + 4 * r, ny * pitch * r + 4 * r,
                                                             nz * pitch * r + 4 * r),
                         gravity=(0.0, 0.0, -9.81), dt=1e-6)
    sc.velocity = rng.normal(0.0, 1.0, size=p.shape)
    sc.angvel = rng.normal(0.0, 300.0, size=p.shape)
    return sc


def _balls_around_cylinder(seed=6):
    """Balls beside a 24 x 8 cylinder mesh (with caps) at distances from
    inside to outside their radius, moving at random: face, edge and vertex
    contacts with the reference's de-duplication."""
    rng = np.random.default_rng(seed)
    mesh = scenes.cylinder_mesh(np.array([0.0, 0, 0]), np.array([0.0, 0, 1]), 0.05, 0.1, 24, 8)
    r = 0.005
    pts = []
    for k in range(160):
        th = rng.uniform(0, 2 * np.pi)
        z = rng.uniform(-0.06, 0.06)  # the mesh spans z in [-0.05, 0.05]: some balls meet the cap edges
        d = 0.05 + r * rng.uniform(0.4, 1.3)
        pts.append([d * np.cos(th), d * np.sin(th), z])
    p = np.array(pts)
    keep = [0]
    for i in range(1, len(p)):  # no two balls overlapping at the start
        if np.min(np.linalg.norm(p[keep] - p[i], axis=1)) > 2.05 * r:
            keep.append(i)
    p = p[keep]
    n = len(p)
    Es, Gs = scenes.hertz_params(1e8, 0.3)
    sc = scenes.DEMScene(name="cylinder_balls", position=p, radius=np.full(n, r), density=np.full(n, 2500.0),
                         material=np.zeros(n, np.int32),
                         hertz=[(0, 0, Es, Gs, 0.8, 0.1, 0.1, 0.3, 0.02, 0.02)],
                         walls=[dict(vertices=mesh["vertices"], tri0=mesh["tri0"], tri1=mesh["tri1"],
                                     tri2=mesh["tri2"], position=(0.0, 0.0, 0.0), material=0)],
                         minb=(-0.08, -0.08, -0.08), maxb=(0.08, 0.08, 0.08), gravity=(0.0, 0.0, 0.0), dt=2e-5)
    sc.velocity = rng.uniform(-0.3, 0.3, size=p.shape)
    sc.angvel = rng.normal(0.0, 20.0, size=p.shape)
    return sc


def _identical_state_forces(torch, ref, sc, prec, k_steps, walls):
    """Runs the reference K steps, loads its state into this library (run K
    steps of its own first, so its lists exist) and compares one force
    evaluation (with the walls and the external hook when asked)."""
    r = ref.RefDEM(sc, torch)
    r.correct_q7 = True
    r.initialize()
    r.step(k_steps)
    g = build_dem(sc, prec)
    g.step(k_steps)
    r.neighbor_search()
    st = r.balls()
    g.setBall(st["pos"], st["vel"], st["angvel"])
    g.neighborSearch()
    a, b = r.pairs(0)
    pg = g.getPairs(0)
    np.testing.assert_array_equal(pg["objectPointed"], a)
    np.testing.assert_array_equal(pg["objectPointing"], b)
    sp = r.springs(0)
    g.importSprings(sp["a"], sp["b"], sp["sliding"], sp["rolling"], sp["torsion"])
    if r.nb:
        bo = r.bonds()
        g.setBondedInteraction(bo["ok"], bo["normal_force"], bo["torsion_torque"], bo["shear_force"],
                               bo["bending_torque"], bo["normal"], bo["point"])
    if walls:
        ws = r.springs(1)
        g.importWallSprings(ws["a"], ws["b"], ws["sliding"], ws["rolling"], ws["torsion"])
    hdt = 0.5 * sc.dt
    r.ball_forces(hdt)
    if walls:
        r.wall_forces(sc.dt)
    r.external(r.time)
    g.evalForces(hdt, walls=walls, wallTimeStep=sc.dt, external=True)
    fr, fg = r.balls(), g.getBall()
    et = torque_err(fg["torque"], fr["torque"], fr["force"], sc.radius)
    return rel_err(fg["force"], fr["force"]), et, r, g


def test_bonds_match_reference_kernels(gpu, ref):
    import torch

    sc = _bonded_block()
    r = ref.RefDEM(sc, torch)
    r.correct_q7 = True  # quirk Q7 (stale reverse ranges) corrected, as in this library
    r.initialize()
    g = build_dem(sc, "fp64")
    bo, bg = r.bonds(), g.getBondedInteraction()
    np.testing.assert_array_equal(bg["objectPointed"], bo["a"])
    np.testing.assert_array_equal(bg["objectPointing"], bo["b"])
    assert rel_err(bg["normal"], bo["normal"]) < 1e-15
    r.step(20)
    g.step(20)
    bo, bg = r.bonds(), g.getBondedInteraction()
    broken = int((bo["ok"] == 0).sum())
    print(f"bonds {len(bo['ok'])}, broken after 20 steps {broken}")
    assert 0 < broken < len(bo["ok"])
    np.testing.assert_array_equal(bg["isBonded"], bo["ok"])
    for k_g, k_r in (("normalForce", "normal_force"), ("shearForce", "shear_force"),
                     ("bendingTorque", "bending_torque"), ("torsionTorque", "torsion_torque"), ("normal", "normal")):
        assert rel_err(bg[k_g], bo[k_r]) < 1e-10, k_g
    st, sg = r.balls(), g.getBall()
    assert rel_err(sg["position"] - sc.position, st["pos"] - sc.position) < 1e-10
    assert rel_err(sg["velocity"], st["vel"]) < 1e-10
    for prec in ("fp64", "mixed"):
        ef, et, r2, _ = _identical_state_forces(torch, ref, sc, prec, 12, walls=False)
        print(f"{prec}: bonded block force {ef:.2e} torque {et:.2e} vs reference kernels")
        assert ef < TOL_STATE[prec] and et < TOL_STATE[prec]


def test_mesh_walls_match_reference_kernels(gpu, ref):
    import torch

    sc = _balls_around_cylinder()
    r = ref.RefDEM(sc, torch)
    r.correct_q7 = True  # quirk Q7 (stale reverse ranges) corrected, as in this library
    r.initialize()
    g = build_dem(sc, "fp64")
    r.step(30)
    g.step(30)
    st, sg = r.balls(), g.getBall()
    a, b = r.pairs(1)
    pw = g.getPairs(1)
    assert len(a) > 20
    assert np.array_equal(np.sort(pair_keys(pw["objectPointed"], pw["objectPointing"])), np.sort(pair_keys(a, b)))
    ev = rel_err(sg["velocity"], st["vel"])
    print(f"{len(a)} ball-triangle pairs; 30 steps FP64 velocity rel err {ev:.2e}")
    assert ev < 1e-10
    assert rel_err(sg["angularVelocity"], st["angvel"]) < 1e-10
    for prec in ("fp64", "mixed"):
        ef, et, _, _ = _identical_state_forces(torch, ref, sc, prec, 15, walls=True)
        print(f"{prec}: wall contact force {ef:.2e} torque {et:.2e} vs reference kernels")
        assert ef < TOL_STATE[prec] and et < TOL_STATE[prec]


def test_buoyancy_drag_matches_reference_kernel(gpu, ref):
    import torch

    sc = scenes.dem_drop(n_side=6, plane_gap=0.002)
    lvl = float(sc.position[:, 2].mean())
    sc.buoyancy = (1000.0, 0.4, (0.0, 0.0, -9.81), (-0.4, 0.1, 0.0), lvl)
    r = ref.RefDEM(sc, torch)
    r.correct_q7 = True  # quirk Q7 (stale reverse ranges) corrected, as in this library
    r.initialize()
    g = build_dem(sc, "fp64")
    r.step(50)
    g.step(50)
    ev = rel_err(g.getBall()["velocity"], r.balls()["vel"])
    print(f"buoyancy + drag: 50 steps FP64 velocity rel err {ev:.2e}")
    assert ev < 1e-10
    for prec in ("fp64", "mixed"):
        ef, _, _, _ = _identical_state_forces(torch, ref, sc, prec, 10, walls=True)
        print(f"{prec}: force with buoyancy + drag {ef:.2e} vs reference kernels")
        assert ef < TOL_STATE[prec]
