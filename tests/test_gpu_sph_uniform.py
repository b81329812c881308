"""The mixed-precision passes specialised for uniform particle constants
(k_sph_accel_u, k_sph_density_u): used for the benchmark scenes, the same
pair sets as the general passes, and the same results within the FP32
rounding of the regrouped terms (the 1e-5 target against FP64 holds
either way)."""
import numpy as np
import pytest

from this_studio_b200 import scenes
from this_studio_b200.scenes import build_sph

from .helpers import oracle_sph, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dam():
    return scenes.dam_break_reference()


def test_uniform_path_selection(gpu, dam):
    assert build_sph(dam, "mixed").uniformKernels()
    assert not build_sph(dam, "fp64").uniformKernels()
    g = build_sph(dam, "mixed")
    g.setUniformKernels(False)
    assert not g.uniformKernels()


def test_uniform_accel_from_identical_state(gpu, oracle_lib, dam):
    o = oracle_sph(dam)
    o.step(40)
    st = o.state()
    o.neighbor_search()
    o.eval_accel()
    ao = o.state()["acc"]
    out = {}
    for uni in (True, False):
        g = build_sph(dam, "mixed")
        g.setUniformKernels(uni)
        g.setSPH(st["pos"], st["vel"], st["rho"], st["p"], st["drho"])
        g.neighborSearch()
        g.evalAcceleration()
        out[uni] = g.getSPH()["acceleration"]
    gv = np.array(dam.gravity)
    e, ei = rel_err(out[True], ao), rel_err(out[True] - gv, ao - gv)
    eg = rel_err(out[True] - gv, out[False] - gv)
    print(f"uniform passes: accel rel err {e:.2e} (interaction {ei:.2e}) vs oracle; {eg:.2e} vs general passes")
    assert e < 1e-5 and ei < 1e-5 and eg < 1e-5


def test_uniform_trajectory_and_pairs(gpu, oracle_lib, dam):
    o = oracle_sph(dam)
    res = {}
    for uni in (True, False):
        g = build_sph(dam, "mixed")
        g.setUniformKernels(uni)
        g.step(60)
        res[uni] = g.getSPH()
        if uni:
            pa = g.getPairs(0)
    o.step(60)
    so = o.state()
    x0 = dam.fluid
    e = rel_err(res[True]["position"] - x0, so["pos"] - x0)
    eg = rel_err(res[True]["position"] - x0, res[False]["position"] - x0)
    er = rel_err(res[True]["density"] - 1000.0, so["rho"] - 1000.0)
    print(f"60 steps: displacement {e:.2e} vs oracle, {eg:.2e} vs general passes; density change {er:.2e}")
    assert e < 1e-5 and eg < 1e-5 and er < 1e-4
    o.neighbor_search()
    ao, bo = o.pairs(0)
    # pair sets at the end state: the mixed state has drifted from the
    # oracle's by FP32 rounding, so compare with exact lists of its own state
    g2 = build_sph(dam, "fp64")
    s = res[True]
    g2.setSPH(s["position"], s["velocity"], s["density"], s["pressure"], s["densityChange"])
    g2.neighborSearch()
    a2, b2 = g2.getPairs(0)
    np.testing.assert_array_equal(pa[0], a2)
    np.testing.assert_array_equal(pa[1], b2)
