"""Device snapshots of a scene's state (demsph_dem_snapshot /
demsph_sph_snapshot): steps from a restored state repeat the steps after the
snapshot bit for bit, and a snapshot restores only into its own scene."""
import numpy as np
import pytest

from this_studio_b200 import _lib, scenes
from this_studio_b200.scenes import build_dem, build_sph

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_dem_snapshot_replays_bit_for_bit(gpu, prec):
    sc = scenes.dem_drop(n_side=10, plane_gap=0.0)
    g = build_dem(sc, prec)
    g.step(13)
    snap = g.snapshot()
    g.step(27)  # across re-sorts and graph blocks
    a = g.getBall()
    pa = g.getPairs(1)
    snap.restore()
    assert g.stepIndex()[0] == 13
    g.step(27)
    b = g.getBall()
    for k in ("position", "velocity", "angularVelocity", "force", "torque"):
        np.testing.assert_array_equal(a[k], b[k])
    np.testing.assert_array_equal(pa["sliding"], g.getPairs(1)["sliding"])
    other = build_dem(sc, prec)
    assert _lib.lib().demsph_dem_restore(other._h, snap._h) == _lib.ERR_INVALID


def test_dem_snapshot_with_bonds(gpu):
    sc = scenes.bonded_beam_clumps(nx=40, ny=4, nz=4, n_clumps=50)
    g = build_dem(sc, "mixed")
    g.step(5)
    snap = g.snapshot()
    g.step(20)
    a, ba = g.getBall(), g.getBondedInteraction()
    snap.restore()
    g.step(20)
    b, bb = g.getBall(), g.getBondedInteraction()
    np.testing.assert_array_equal(a["position"], b["position"])
    np.testing.assert_array_equal(ba["normalForce"], bb["normalForce"])
    np.testing.assert_array_equal(g.getClump()["orientation"], g.getClump()["orientation"])


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_sph_snapshot_replays_bit_for_bit(gpu, prec):
    sc = scenes.dam_break_reference()
    g = build_sph(sc, prec)
    g.step(11)
    snap = g.snapshot()
    g.step(30)
    a = g.getSPH()
    snap.restore()
    assert g.stepIndex()[0] == 11
    g.step(30)
    b = g.getSPH()
    for k in ("position", "velocity", "density", "pressure", "densityChange"):
        np.testing.assert_array_equal(a[k], b[k])
