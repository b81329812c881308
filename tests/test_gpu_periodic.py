"""Periodic boundaries (setPeriodicBoundary) on the GPU against the oracle's
restatement of the reference's ghost passes (addDummyContactForceTorque,
DEMSolver.h:279-426): the ghost pair sets of every active direction, their
springs and forces, and a short trajectory.

The scene tiles the box exactly, so the reference's rules show: a ghost pair
needs the querying ball's index below the ghost's, so contacts across a face
between a low-index ghost and a high-index ball are not found, and two ghosts
shifted together reproduce a contact the main list already holds."""
import numpy as np
import pytest

from this_studio_b200 import scenes

from .helpers import oracle_dem, rel_err

pytestmark = pytest.mark.gpu

SETS = ("X", "Y", "Z", "XY", "YZ", "XZ", "XYZ")


def _keyed(a, b, v):
    return {(int(x), int(y)): v[k] for k, (x, y) in enumerate(zip(a, b))}


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-11), ("mixed", 1e-5)])
def test_ghost_pairs_and_forces_match_oracle(gpu, oracle_lib, prec, tol):
    sc = scenes.dem_periodic_box(n_side=8, periodic=(True, True, True))
    o = oracle_dem(sc)
    g = scenes.build_dem(sc, prec)
    o.step(3)
    g.step(3)
    for k, name in enumerate(SETS):
        po = o.ghost_pairs(k)
        pg = g.getPairs(2 + k)
        assert len(po["a"]) > 0
        ko = _keyed(po["a"], po["b"], po["force"])
        kg = _keyed(pg["objectPointed"], pg["objectPointing"], pg["force"])
        assert set(ko) == set(kg), name
        keys = sorted(ko)
        fo = np.array([ko[q] for q in keys])
        fg = np.array([kg[q] for q in keys])
        e = rel_err(fg, fo)
        print(f"{prec} ghost set {name}: {len(keys)} pairs, force rel err {e:.2e}")
        assert e < tol


def test_periodic_trajectory_matches_oracle(gpu, oracle_lib):
    sc = scenes.dem_periodic_box(n_side=8, periodic=(True, True, False))
    o = oracle_dem(sc)
    g = scenes.build_dem(sc, "fp64")
    o.step(40)
    g.step(40)
    so, sg = o.balls(), g.getBall()
    e = rel_err(sg["position"] - sc.position, so["pos"] - sc.position)
    ev = rel_err(sg["velocity"], so["vel"])
    print(f"periodic XY, 40 steps: displacement rel err {e:.2e}, velocity {ev:.2e}")
    assert e < 1e-9 and ev < 1e-9


def test_ghost_passes_match_reference_kernels(gpu):
    """One evaluation with every ghost pass, from fresh lists, against the
    reference's own launchers (launchBuildDummyPosition,
    launchUpdateDummySpatialGridCellHashStartEnd, the ball pair and contact
    kernels) built from its sources: identical ghost pairs, ball forces."""
    import torch

    from oracle import ref_harness as ref

    if not ref.available():
        pytest.skip("the reference's CUDA build is not present")
    sc = scenes.dem_periodic_box(n_side=8, periodic=(True, True, True))
    g = scenes.build_dem(sc, "fp64")
    g.neighborSearch()
    g.evalForces(1e-5, periodic=True)
    r = ref.RefDEMPairs(sc, torch)
    r.neighbor_search()
    r.forces(1e-5)
    dirs = ((1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (0, 1, 1), (1, 0, 1), (1, 1, 1))
    for k, d in enumerate(dirs):
        a, b, f = r.ghost_pass(d, 1e-5)
        pg = g.getPairs(2 + k)
        assert sorted(zip(a.tolist(), b.tolist())) == sorted(zip(pg["objectPointed"].tolist(),
                                                                 pg["objectPointing"].tolist())), SETS[k]
    fr, tr = r.force.cpu().numpy(), r.torque.cpu().numpy()
    gb = g.getBall()
    ef, et = rel_err(gb["force"], fr), rel_err(gb["torque"], tr)
    print(f"ghost passes vs reference kernels: force {ef:.2e}, torque {et:.2e}")
    assert ef < 1e-12 and et < 1e-11
