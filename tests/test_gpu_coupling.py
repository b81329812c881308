"""Particle-level DEM-SPH coupling on the GPU against the oracle's
restatement: marker placement, one coupled step (fluid state, the force
and torque on each ball, the balls' state), a trajectory of coupled steps in
FP64 and mixed precision, fluid steps alone with the markers frozen, exact
momentum exchange, and the argument checks of the C ABI."""
import numpy as np
import pytest

from this_studio_b200 import DemsphError, scenes

from .helpers import coupled_momentum, oracle_coupled, rel_err
from .test_coupling_oracle import hydrostatic

pytestmark = pytest.mark.gpu

BALLS = ((0.5, 0.5, 0.45, 4.0, 1200.0), (0.25, 0.3, 0.7, 2.5, 600.0), (0.75, 0.7, 0.3, 3.0, 2500.0))


def _scene(**kw):
    args = dict(nx=16, ny=16, depth=16, balls=BALLS, ball_velocity=[[0.1, 0, -0.2], [0, 0.3, 0.1], [-0.2, 0, 0]])
    args.update(kw)
    sc = scenes.balls_in_tank(**args)
    sc.dem.angvel = np.array([[0.0, 0.0, 4.0], [3.0, 0.0, 0.0], [0.0, -2.0, 1.0]])
    return sc


def _pair(sc, prec):
    o_f, o_d = oracle_coupled(sc)
    g_f, g_d, cpl = scenes.build_coupled(sc, prec)
    rho, p, drho = hydrostatic(sc)
    o_f.set_state(rho=rho, p=p, drho=drho)
    g_f.setSPH(density=rho, pressure=p, densityChange=drho)
    return o_f, o_d, g_f, g_d, cpl


def test_markers_match_oracle(gpu, oracle_lib):
    sc = _scene()
    o_f, o_d, g_f, g_d, cpl = _pair(sc, "fp64")
    mo, mg = o_f.markers(), cpl.getMarkers()
    assert cpl.numMarkers() == (len(mo["ball"]), 3)
    assert np.array_equal(mo["ball"], mg["ball"])
    for a, b in (("pos", "position"), ("vel", "velocity"), ("normal", "normal")):
        assert np.allclose(mg[b], mo[a], rtol=0, atol=1e-14), a


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-11), ("mixed", 1e-5)])
def test_one_coupled_step_matches_oracle(gpu, oracle_lib, prec, tol):
    sc = _scene()
    o_f, o_d, g_f, g_d, cpl = _pair(sc, prec)
    o_f.couple_step(o_d, 1, sc.dem_substeps)
    cpl.step(1, sc.dem_substeps)
    bo, Fo, To = o_f.coupling(o_d, 3)
    bg, Fg, Tg = cpl.getForces()
    assert np.array_equal(bo, bg)
    ef, et = rel_err(Fg, Fo), rel_err(Tg, To)
    mo = o_f.markers()["force"]
    em = rel_err(cpl.getMarkers()["force"], mo)
    so, sg = o_f.state(), g_f.getSPH()
    ea = rel_err(sg["acceleration"], so["acc"])
    ev = rel_err(sg["velocity"], so["vel"])
    er = rel_err(sg["density"] - sc.sph.density, so["rho"] - sc.sph.density)
    bo_, bg_ = o_d.balls(), g_d.getBall()
    eb = rel_err(bg_["velocity"], bo_["vel"])
    ew = rel_err(bg_["angularVelocity"], bo_["angvel"])
    print(f"{prec}: ball force {ef:.2e} torque {et:.2e} marker reactions {em:.2e} fluid acc {ea:.2e} "
          f"vel {ev:.2e} drho {er:.2e} ball vel {eb:.2e} omega {ew:.2e}")
    for e in (ef, et, em, ea, ev, er, eb, ew):
        assert e < tol


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-5)])
def test_coupled_trajectory_matches_oracle(gpu, oracle_lib, prec, tol):
    """Twenty coupled steps: displacements, ball velocities and the last
    step's force on the balls within the target's 1e-5 (mixed) of the FP64
    oracle."""
    sc = _scene()
    o_f, o_d, g_f, g_d, cpl = _pair(sc, prec)
    o_f.couple_step(o_d, 20, sc.dem_substeps)
    cpl.step(20, sc.dem_substeps)
    so, sg = o_f.state(), g_f.getSPH()
    bo, bg = o_d.balls(), g_d.getBall()
    x0 = sc.sph.fluid
    ep = rel_err(sg["position"] - x0, so["pos"] - x0)
    ebp = rel_err(bg["position"] - sc.dem.position, bo["pos"] - sc.dem.position)
    ebv = rel_err(bg["velocity"], bo["vel"])
    _, Fo, _ = o_f.coupling(o_d, 3)
    _, Fg, _ = cpl.getForces()
    ef = rel_err(Fg, Fo)
    print(f"{prec}, 20 coupled steps: fluid displacement {ep:.2e} ball displacement {ebp:.2e} "
          f"ball vel {ebv:.2e} force {ef:.2e}")
    assert ep < tol and ebp < tol and ebv < tol and ef < tol


def test_fluid_steps_alone_keep_markers(gpu, oracle_lib):
    """Stepping the fluid alone after a coupled step: the markers stay where
    the coupled step left them and act as dummies."""
    sc = _scene()
    o_f, o_d, g_f, g_d, cpl = _pair(sc, "fp64")
    o_f.couple_step(o_d, 2, sc.dem_substeps)
    cpl.step(2, sc.dem_substeps)
    o_f.step(3)
    g_f.step(3)
    so, sg = o_f.state(), g_f.getSPH()
    e = rel_err(sg["position"] - sc.sph.fluid, so["pos"] - sc.sph.fluid)
    assert e < 1e-10
    assert np.allclose(cpl.getMarkers()["position"], o_f.markers()["pos"], rtol=0, atol=1e-13)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_momentum_exchange_is_exact(gpu, oracle_lib, prec, tol):
    """No gravity, no walls: total momentum of the fluid and the balls is
    conserved to rounding (in FP64 to the last bits; in mixed precision to
    the FP32 rounding of the fluid's summed accelerations)."""
    v0 = np.array([[0.8, -0.3, 0.2]])
    sc = scenes.balls_in_tank(nx=14, ny=14, depth=14, balls=((0.5, 0.5, 0.5, 3.0, 800.0),), ball_velocity=v0,
                              gravity=(0.0, 0.0, 0.0), walls=False)
    f, d, cpl = scenes.build_coupled(sc, prec)
    p0 = coupled_momentum(sc, np.zeros((len(sc.sph.fluid), 3)), v0)
    cpl.step(6, sc.dem_substeps)
    p1 = coupled_momentum(sc, f.getSPH()["velocity"], d.getBall()["velocity"])
    mb = sc.dem.density[0] * (4.0 / 3.0) * np.pi * sc.dem.radius[0] ** 3
    drift = np.linalg.norm(p1 - p0) / (mb * np.linalg.norm(v0))
    print(f"{prec}: momentum drift over 6 coupled steps {drift:.2e}")
    assert drift < tol


def test_argument_checks(gpu):
    sc = _scene()
    f, d, cpl = scenes.build_coupled(sc, "fp64")
    with pytest.raises(DemsphError):
        cpl.step(1, sc.dem_substeps + 1)  # DEM dt x substeps != fluid dt
    with pytest.raises(DemsphError):
        cpl.addBalls([0], sc.marker_spacing, sc.marker_h, 10.0, 1e-3, 1000.0)  # coupled twice
    with pytest.raises(DemsphError):
        cpl.addBalls([7], sc.marker_spacing, sc.marker_h, 10.0, 1e-3, 1000.0)  # no such ball
    with pytest.raises(DemsphError):
        cpl.addBalls([1], sc.marker_spacing, 10.0, 10.0, 1e-3, 1000.0)  # h above the fluid's
    other = scenes.build_dem(sc.dem, "fp64")
    from this_studio_b200 import DEMSPHCoupling

    with pytest.raises(DemsphError):
        DEMSPHCoupling(f, other).step(1, sc.dem_substeps)
    cpl.step(1, sc.dem_substeps)  # still usable after the refused calls


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_graph_replay_matches_direct_launches(gpu, prec):
    """Coupled steps replayed from CUDA graphs (blocks of ten) give the same
    bits as the same steps launched one kernel at a time."""
    sc = _scene()
    runs = []
    for graphs in (True, False):
        f, d, cpl = scenes.build_coupled(sc, prec)
        f.setGraphs(graphs)
        d.setGraphs(graphs)
        cpl.step(7, sc.dem_substeps)   # eager up to the DEM re-sort, then part of a block
        cpl.step(23, sc.dem_substeps)  # two blocks and a tail
        runs.append((f.getSPH(), d.getBall(), cpl.getForces()))
    (fa, ba, ca), (fb, bb, cb) = runs
    assert np.array_equal(fa["position"], fb["position"])
    assert np.array_equal(fa["velocity"], fb["velocity"])
    assert np.array_equal(fa["density"], fb["density"])
    assert np.array_equal(ba["position"], bb["position"])
    assert np.array_equal(ba["angularVelocity"], bb["angularVelocity"])
    assert np.array_equal(ca[1], cb[1]) and np.array_equal(ca[2], cb[2])
    assert f.stepIndex()[0] == 30 and d.stepIndex()[0] == 30 * sc.dem_substeps


def test_balls_float_near_their_flotation_height(gpu):
    """Physical check of the coupling (it has no reference counterpart): two
    balls of density 500 and 800 released in still water bob and settle
    (about six bobbing periods, 24,000 steps); their mean heights over the
    last third sit within 0.5 R of the static flotation height of a sphere
    (submerged cap volume = its mass / rho_water, the reference's
    waterSurfaceHeightForStaticSphere) above the water level raised by the
    balls' displaced volume, and the denser ball sits lower by the analytic
    difference to within 0.25 R."""
    balls = ((0.3, 0.5, 0.85, 4.0, 500.0), (0.7, 0.5, 0.85, 4.0, 800.0))
    sc = scenes.balls_in_tank(nx=40, ny=32, depth=24, balls=balls, dem_substeps=1)
    f, d, c = scenes.build_coupled(sc, "mixed")
    rho, p, drho = hydrostatic(sc)
    f.setSPH(density=rho, pressure=p, densityChange=drho)
    R = sc.dem.radius
    H = sc.sph.fluid[:, 2].max() + 0.5 * sc.sph.spacing
    area = (40 * sc.sph.spacing) * (32 * sc.sph.spacing)
    expect = []
    for r, (_, _, _, _, rho_b) in zip(R, balls):
        h = scenes.static_sphere_water_level(r, rho_b, 1000.0)  # water plane above the centre
        expect.append(H - h)
    rise = sum(rb / 1000.0 * 4.0 / 3.0 * np.pi * r ** 3 for r, (_, _, _, _, rb) in zip(R, balls)) / area
    expect = np.array(expect) + rise
    zs = []
    for _ in range(60):
        c.step(400, 1)
        zs.append(d.getBall()["position"][:, 2].copy())
    zs = np.array(zs)
    mean = zs[40:].mean(axis=0)
    print(f"settled centres {mean}, static flotation {expect} (R {R[0]:.3f}); "
          f"offsets {(mean - expect) / R} R; difference {mean[0] - mean[1]:.4f} vs {expect[0] - expect[1]:.4f}")
    assert np.all(np.abs(mean - expect) < 0.5 * R)
    assert abs((mean[0] - mean[1]) - (expect[0] - expect[1])) < 0.25 * R[0]


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("mixed", 1e-5)])
def test_ice_sheet_form_coupled_step(gpu, oracle_lib, prec, tol):
    """The coupled ice-sheet workload's form at a size the oracle runs in a
    moment: a hexagonal sheet of 672 jittered Hertz-Mindlin spheres bonded at
    their initial contacts (parallel bonds), moving at 0.5 m/s towards a
    cylinder mesh, one centre marker per sphere, floating half submerged on a
    two-layer water film over a dummy floor at hydrostatic pressure.  One
    coupled step from the same state: the bond set, the balls' force and
    torque (contacts, bonds, coupling and gravity), the coupling force on the
    balls and the fluid's acceleration against the FP64 oracle."""
    from .helpers import torque_err

    sc = scenes.ice_sheet_on_water(n_side=24, fluid=8000, cyl_segments=(24, 6))
    n = sc.dem.position.shape[0]
    o_f, o_d = oracle_coupled(sc)
    g_f, g_d, cpl = scenes.build_coupled(sc, prec)
    rho, p, drho = hydrostatic(sc)
    o_f.set_state(rho=rho, p=p, drho=drho)
    g_f.setSPH(density=rho, pressure=p, densityChange=drho)
    ob, gb = o_d.bonds(), g_d.getBondedInteraction()
    assert len(ob["a"]) > n
    keys = lambda a, b: np.unique(np.minimum(a, b).astype(np.int64) * n + np.maximum(a, b))
    assert np.array_equal(keys(ob["a"], ob["b"]), keys(gb["objectPointed"], gb["objectPointing"]))
    o_f.couple_step(o_d, 1, sc.dem_substeps)
    cpl.step(1, sc.dem_substeps)
    bo, bg = o_d.balls(), g_d.getBall()
    ef = rel_err(bg["force"], bo["force"])
    et = torque_err(bg["torque"], bo["torque"], bo["force"], sc.dem.radius)
    _, Fo, _ = o_f.coupling(o_d, n)
    _, Fg, _ = cpl.getForces()
    ec = rel_err(Fg, Fo)
    ea = rel_err(g_f.getSPH()["acceleration"], o_f.state()["acc"])
    print(f"{prec}: ice sheet form, {n} spheres, {len(ob['a'])} bonds: ball force {ef:.2e} torque {et:.2e} "
          f"coupling force {ec:.2e} fluid acc {ea:.2e}")
    for e in (ef, et, ec, ea):
        assert e < tol
