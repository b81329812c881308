"""Parity at the sizes the benchmark reports.

* WCSPH dam break, 128,000 fluid particles and 150,216 dummy wall particles
  (the bench workload): fluid-fluid, fluid-dummy and dummy-dummy pair sets
  identical to the reference's own kernels (built from its sources,
  oracle/ref_harness.RefSPH), and the acceleration of one evaluation from an
  identical state against the reference kernels, in FP64 and in mixed
  precision.
* DEM bounce, 4,096 Hertz-Mindlin spheres on the 2-triangle plane, in its
  contact-rich form (plane touching the lowest sphere, run until the bottom
  layer presses on it), and the same 4,096 spheres as a touching pack with
  friction, rolling and torsion: one force evaluation from an identical state
  against the FP64 oracle.
* Bonded beam (20 x 20 x 400 spheres, 462,840 parallel bonds) plus 20,000
  three-sphere clumps: one force evaluation from an identical state (balls,
  contact springs and bond state) against the FP64 oracle.

Tolerances: the force error is ||F - F64|| / ||F64|| over all particles,
the torque error ||T - T64|| / max(||T64||, ||F64|| r_mean) (the torques
of spheres pressed straight onto a plane vanish to rounding, so they are
measured against the torque scale of the forces): at most 1e-5 in mixed
precision (FP32 force arithmetic, the target's bound) and 1e-10 in FP64
(the reference's arithmetic; rounding only).
"""
import numpy as np
import pytest

from this_studio_b200 import scenes
from this_studio_b200.scenes import build_dem, build_sph

from .helpers import oracle_dem, pair_keys, rel_err, torque_err

pytestmark = pytest.mark.gpu
TOL = {"fp64": 1e-10, "mixed": 1e-5}


@pytest.fixture(scope="module")
def ref():
    from oracle import ref_harness

    if not ref_harness.available():
        pytest.skip("oracle/_ref/libdemsph_ref.so not built (make -f oracle/Makefile.ref)")
    return ref_harness


@pytest.fixture(scope="module")
def dam128k():
    return scenes.sph_dam_break()


@pytest.fixture(scope="module")
def dam128k_ref_state(gpu, ref, dam128k):
    """The reference kernels' state after 25 steps of the 128k dam break
    (the column has started to fall and spread), its pair lists rebuilt
    at that state, and the acceleration of one evaluation there."""
    import torch

    r = ref.RefSPH(dam128k, torch)
    r.step(25)
    r.neighbor_search()
    st = r.state()
    pairs = [r.pairs(w) for w in (0, 1, 2)]
    r._half(False)  # momentum at the state (then kick + drift, not used)
    acc = r.state()["acc"]
    del r
    torch.cuda.empty_cache()
    return st, pairs, acc


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_dam_break_128k_pairs_and_accel_match_reference_kernels(gpu, dam128k, dam128k_ref_state, prec):
    st, pairs, acc = dam128k_ref_state
    g = build_sph(dam128k, prec)
    assert g.num() == 128_000 and g.num(dummy=True) == 150_216
    # dummy-dummy pairs of the wall-normal initialisation
    a, b = g.getPairs(2)
    np.testing.assert_array_equal(a, pairs[2][0])
    np.testing.assert_array_equal(b, pairs[2][1])
    g.setSPH(st["pos"], st["vel"], st["rho"], st["p"], st["drho"])
    g.neighborSearch()
    for w in (0, 1):
        a, b = g.getPairs(w)
        assert len(a) == len(pairs[w][0])
        np.testing.assert_array_equal(a, pairs[w][0])
        np.testing.assert_array_equal(b, pairs[w][1])
    print(f"pairs: fluid-fluid {len(pairs[0][0])}, fluid-dummy {len(pairs[1][0])}, dummy-dummy {len(pairs[2][0])}")
    g.evalAcceleration()
    ag = g.getSPH()["acceleration"]
    gvec = np.array(dam128k.gravity)
    e, ei = rel_err(ag, acc), rel_err(ag - gvec, acc - gvec)
    print(f"{prec}: 128k acceleration rel err {e:.3e} (interaction part {ei:.3e}) vs reference kernels")
    assert e < TOL[prec] and ei < TOL[prec]


def _oracle_identical_state(sc, prec, k_steps, walls, const_force=None):
    """Oracle K steps; this library K steps of its own (so its lists exist),
    then the oracle's balls, contact springs, wall springs and bond state
    loaded into it; one force evaluation on both sides."""
    o = oracle_dem(sc)
    if const_force is not None:
        o.set_constant_force(const_force)
    o.step(k_steps)
    g = build_dem(sc, prec)
    g.step(k_steps)
    bo = o.balls()
    g.setBall(bo["pos"], bo["vel"], bo["angvel"])
    o.neighbor_search()
    g.neighborSearch()
    po, pg = o.pairs(0), g.getPairs(0)
    np.testing.assert_array_equal(pg["objectPointed"], po["a"])
    np.testing.assert_array_equal(pg["objectPointing"], po["b"])
    g.importSprings(po["a"], po["b"], po["sliding"], po["rolling"], po["torsion"])
    if o.bonds()["a"].size:
        b = o.bonds()
        g.setBondedInteraction(b["ok"], b["normal_force"], b["torsion_torque"], b["shear_force"],
                               b["bending_torque"], b["normal"], b["point"])
    if walls:
        wo, wg = o.pairs(1), g.getPairs(1)
        # the wall rows carry history by (ball, triangle): every oracle row is one of ours
        assert set(pair_keys(wo["a"], wo["b"])) <= set(pair_keys(wg["objectPointed"], wg["objectPointing"]))
        g.importWallSprings(wo["a"], wo["b"], wo["sliding"], wo["rolling"], wo["torsion"])
    hdt = 0.5 * sc.dt
    o.eval_forces(hdt, walls=walls, dt_wall=sc.dt)
    g.evalForces(hdt, walls=walls, wallTimeStep=sc.dt)
    fo, fg = o.balls(), g.getBall()
    et = torque_err(fg["torque"], fo["torque"], fo["force"], sc.radius)
    return rel_err(fg["force"], fo["force"]), et, o, g


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_bounce_4096_contact_rich_forces(gpu, oracle_lib, prec):
    """The plain DEM bounce (4,096 spheres, r 5 mm, Hertz-Mindlin E 1e8,
    nu 0.3, e 0.8, mu 0.3, dt 1e-5) with the plane touching the lowest
    sphere: over the 1,000 steps of the workload the bottom layer falls onto
    the plane (the lattice keeps the spheres 2 mm apart, so the contacts are
    sphere-plane)."""
    sc = scenes.dem_drop(plane_gap=0.0)
    assert sc.position.shape[0] == 4096
    ef, et, o, g = _oracle_identical_state(sc, prec, 1000, walls=True)
    nw = len(o.pairs(1)["a"])
    touching = int((np.linalg.norm(o.balls()["force"], axis=1) > 0).sum())
    print(f"{prec}: 4096 bounce, {nw} wall rows, {touching} balls in contact: force {ef:.2e} torque {et:.2e}")
    assert touching >= 10
    assert ef < TOL[prec] and et < TOL[prec]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_pack_4096_forces(gpu, oracle_lib, prec):
    sc = scenes.dem_pack(n_side=16)
    ef, et, o, _ = _oracle_identical_state(sc, prec, 12, walls=False)
    print(f"{prec}: 4096 pack, {len(o.pairs(0)['a'])} pairs: force {ef:.2e} torque {et:.2e}")
    assert ef < TOL[prec] and et < TOL[prec]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_beam_and_clumps_forces(gpu, oracle_lib, prec):
    sc = scenes.bonded_beam_clumps()
    ef, et, o, g = _oracle_identical_state(sc, prec, 20, walls=False, const_force=sc.constant_force)
    nb = len(o.bonds()["a"])
    print(f"{prec}: beam + clumps, {o.num_balls} spheres, {nb} bonds: force {ef:.2e} torque {et:.2e}")
    assert nb == 462_840
    assert ef < TOL[prec] and et < TOL[prec]
