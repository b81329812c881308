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


def test_uniform_passes_with_markers(gpu, oracle_lib):
    """A coupled scene (uniform fluid and dummy constants, markers on three
    balls) runs the specialised passes with unpacked shadows: 20 coupled
    steps give the same ball forces, fluid and ball trajectories as the
    general passes within the FP32 rounding of the regrouped terms, and both
    stay within the 1e-5 target of the FP64 oracle."""
    from .helpers import oracle_coupled
    from .test_coupling_oracle import hydrostatic

    balls = ((0.5, 0.5, 0.45, 4.0, 1200.0), (0.25, 0.3, 0.7, 2.5, 600.0), (0.75, 0.7, 0.3, 3.0, 2500.0))
    sc = scenes.balls_in_tank(nx=16, ny=16, depth=16, balls=balls,
                              ball_velocity=[[0.1, 0, -0.2], [0, 0.3, 0.1], [-0.2, 0, 0]])
    rho, p, drho = hydrostatic(sc)
    o_f, o_d = oracle_coupled(sc)
    o_f.set_state(rho=rho, p=p, drho=drho)
    o_f.couple_step(o_d, 20, sc.dem_substeps)
    _, Fo, _ = o_f.coupling(o_d, 3)
    res = {}
    for uni in (True, False):
        f, d, c = scenes.build_coupled(sc, "mixed")
        f.setUniformKernels(uni)
        f.setSPH(density=rho, pressure=p, densityChange=drho)
        assert f.uniformKernels() == uni
        c.step(20, sc.dem_substeps)
        res[uni] = (f.getSPH()["position"], d.getBall()["position"], c.getForces()[1])
    x0, b0 = sc.sph.fluid, sc.dem.position
    ep = rel_err(res[True][0] - x0, res[False][0] - x0)
    eb = rel_err(res[True][1] - b0, res[False][1] - b0)
    ef = rel_err(res[True][2], res[False][2])
    eo = rel_err(res[True][2], Fo)
    eop = rel_err(res[True][0] - x0, o_f.state()["pos"] - x0)
    print(f"coupled, uniform vs general passes: fluid displacement {ep:.2e} ball displacement {eb:.2e} "
          f"force {ef:.2e}; uniform vs oracle: force {eo:.2e} fluid displacement {eop:.2e}")
    assert ep < 1e-5 and eb < 1e-5 and ef < 1e-5
    assert eo < 1e-5 and eop < 1e-5
