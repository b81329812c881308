"""Skin lists: a fluid step that reuses rows built with a skin and keeps the
pairs within the exact cutoff uses the reference's per-step pair set.
Checked step by step against scenes that rebuild exact lists every step, in
both precisions, with the rebuilds counted; graph replay against direct
launches; the setting's limits."""
import numpy as np
import pytest

from this_studio_b200 import DemsphError, scenes
from this_studio_b200.scenes import build_sph
from this_studio_b200.solvers import WCSPHSolver

from .helpers import rel_err

pytestmark = pytest.mark.gpu


def _build(sc, prec, skin):
    s = WCSPHSolver()
    s.setSkin(skin)
    s.addSPHs(sc.fluid, None, sc.sound_speed, sc.spacing, sc.density, sc.viscosity)
    s.addDummies(sc.dummy, None, sc.sound_speed, sc.spacing, sc.density, sc.viscosity)
    s.initialize(sc.minb, sc.maxb, sc.gravity, sc.dt, prec)
    return s


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_skin_steps_use_the_exact_pair_set(gpu, prec):
    sc = scenes.dam_break_reference()
    a = _build(sc, prec, 0.05)
    b = _build(sc, prec, 0.0)
    assert a.skinStats()[0] == pytest.approx(0.05)
    assert b.skinStats()[0] == 0.0
    for k in range(40):
        a.step(1)
        b.step(1)
        for w in (0, 1):
            pa, pb = a.getPairs(w), b.getPairs(w)
            assert len(pa[0]) == len(pb[0]), (k, w)
            np.testing.assert_array_equal(pa[0], pb[0])
            np.testing.assert_array_equal(pa[1], pb[1])
    fa, fb = a.getSPH(), b.getSPH()
    e = rel_err(fa["position"] - sc.fluid, fb["position"] - sc.fluid)
    ev = rel_err(fa["velocity"], fb["velocity"])
    rebuilds = a.skinStats()[1]
    print(f"{prec}: 40 steps, {rebuilds} skin rebuilds; displacement {e:.2e}, velocity {ev:.2e} vs exact lists")
    assert 1 <= rebuilds < 40
    assert e < (1e-12 if prec == "fp64" else 1e-6) and ev < (1e-11 if prec == "fp64" else 1e-5)


def test_skin_graph_replay_matches_direct_launches(gpu):
    """The gated rebuild inside captured steps gives the same bits as direct launches."""
    sc = scenes.dam_break_reference()
    out = []
    for graphs in (True, False):
        s = _build(sc, "mixed", 0.05)
        s.setGraphs(graphs)
        s.step(37)
        out.append((s.getSPH(), s.skinStats()[1]))
    (sa, ra), (sb, rb) = out
    assert ra == rb
    for k in ("position", "velocity", "density", "pressure"):
        np.testing.assert_array_equal(sa[k], sb[k])


def test_skin_setting(gpu):
    sc = scenes.dam_break_reference()
    s = _build(sc, "fp64", 0.1)
    with pytest.raises(DemsphError):
        s.setSkin(0.2)  # above what the grid was built for
    s.setSkin(0.05)
    s.step(5)
    s.setSkin(0.0)
    s.step(5)
    assert s.skinStats()[0] == 0.0


def test_tune_skin_restores_the_state(gpu):
    """The skin tuner times steps from a saved state and puts it back: the
    scene after tuning steps on as one that was never tuned (to rounding, as
    the skin sets the order in which pairs are summed), in mixed precision,
    whose FP32 and fixed-point copies must follow the restored records."""
    sc = scenes.dam_break_reference()
    a = _build(sc, "mixed", 0.05)
    b = _build(sc, "mixed", 0.05)
    a.step(10)
    b.step(10)
    before = a.getSPH()
    chosen, ms = a.tuneSkin(8)
    assert chosen in (0.0, pytest.approx(0.025), pytest.approx(0.05))
    assert all(m > 0 for m in ms)
    assert a.stepIndex()[0] == 10
    np.testing.assert_array_equal(a.getSPH()["position"], before["position"])
    a.step(20)
    b.step(20)
    for w in (0, 1):
        pa, pb = a.getPairs(w), b.getPairs(w)
        np.testing.assert_array_equal(pa[0], pb[0])
        np.testing.assert_array_equal(pa[1], pb[1])
    fa, fb = a.getSPH(), b.getSPH()
    e = rel_err(fa["position"] - sc.fluid, fb["position"] - sc.fluid)
    print(f"tuned skin {chosen} ({', '.join(f'{m:.3f}' for m in ms)} ms/step); displacement vs untuned {e:.2e}")
    assert e < 1e-6


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_coupled_skin_steps_match_exact_lists(gpu, prec):
    """Coupled steps on skin rows (the fluid-marker rows and their transposed
    rows are rebuilt with the fluid's, when a fluid particle or a marker has
    drifted half the skin) against the same steps on exact lists rebuilt
    every step: fast balls make the markers' drift force most rebuilds."""
    sc = scenes.balls_in_tank(nx=16, ny=16, depth=16, balls=((0.5, 0.5, 0.45, 4.0, 1200.0), (0.25, 0.3, 0.7, 2.5, 600.0)),
                              ball_velocity=[[1.5, 0.0, -1.0], [0.0, 2.0, 0.5]])
    runs = []
    for skin in (0.04, 0.0):  # the default skin, then exact lists every step
        f, d, cpl = scenes.build_coupled(sc, prec)
        f.setSkin(skin)
        cpl.step(7, sc.dem_substeps)
        cpl.step(33, sc.dem_substeps)
        runs.append((f.getSPH(), d.getBall(), cpl.getForces(), f.skinStats()[1]))
    (fa, ba, ca, ra), (fb, bb, cb, rb) = runs
    e = rel_err(fa["position"] - sc.sph.fluid, fb["position"] - sc.sph.fluid)
    ev = rel_err(fa["velocity"], fb["velocity"])
    eb = rel_err(ba["position"] - sc.dem.position, bb["position"] - sc.dem.position)
    ef = rel_err(ca[1], cb[1])
    print(f"{prec}: 40 coupled steps, {ra} skin rebuilds; fluid displacement {e:.2e}, velocity {ev:.2e}, "
          f"ball displacement {eb:.2e}, ball force {ef:.2e} vs exact lists")
    assert 8 <= ra < 40
    tol = 1e-10 if prec == "fp64" else 2e-5
    assert e < tol and ev < tol and eb < tol and ef < 10 * tol


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_conditional_rebuild_matches_gated_launches(gpu, prec):
    """Graph steps whose rebuild is a conditional node give the same bits as
    graph steps that launch the gated rebuild every step and as direct
    launches, with the same rebuilds; a second scene on the same lists after a
    snapshot / restore does too."""
    sc = scenes.dam_break_reference()
    out = []
    for cond, graphs in ((True, True), (False, True), (False, False)):
        s = _build(sc, prec, 0.05)
        s.setConditionalRebuild(cond)
        s.setGraphs(graphs)
        s.step(37)
        active, per = s.conditionalRebuild()
        assert active == (cond and graphs)
        if active:
            assert per > 0
        snap = s.snapshot()
        s.step(11)
        snap.restore()
        s.step(11)
        out.append((s.getSPH(), s.skinStats()[1]))
    (s0, r0) = out[0]
    for s1, r1 in out[1:]:
        assert r1 == r0
        for k in ("position", "velocity", "density", "pressure"):
            np.testing.assert_array_equal(s0[k], s1[k])
    print(f"{prec}: {r0} rebuilds over 59 steps, identical with and without conditional nodes")


def test_list_overflow_regrows_at_the_next_call(gpu):
    """Rows sized with no headroom overflow once the fluid is compressed: the
    passes walk those particles' stencils (same pairs), the step call returns
    without waiting, and the next call regrows the lists from the status the
    steps left.  The trajectory matches a scene whose rows had room."""
    sc = scenes.dam_break_reference()
    a = build_sph(sc, "fp64", configure=lambda s: s.setListHeadroom(0.0))
    b = build_sph(sc, "fp64", configure=lambda s: s.setListHeadroom(1.0))
    c = sc.fluid.mean(axis=0)
    # 10% closer: the lattice's next shells of neighbours move inside the
    # cutoff and the skin (a few percent would add none: the shell radii are
    # square roots of sums of three squares)
    squeezed = c + 0.9 * (sc.fluid - c)
    for s in (a, b):
        s.setSPH(position=squeezed)
    k0 = a.listCapacity()
    for _ in range(5):
        a.step(6)
        b.step(6)
    a.synchronize()
    k1 = a.listCapacity()
    print(f"row capacity {k0} -> {k1} (room: {b.listCapacity()})")
    assert k1[0] > k0[0]
    e = rel_err(a.getSPH()["position"] - squeezed, b.getSPH()["position"] - squeezed)
    print(f"30 steps, lists regrown vs rows with room: displacement {e:.2e}")
    assert e < 1e-9
