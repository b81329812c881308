"""Batched and served forms.

CPU: tile packing.  GPU: a scene gives the same result alone and inside a
batch whose membership changes while it runs (the batched form's contract),
and the server completes a small stream with the results of each scene equal
to running it alone."""
import numpy as np
import pytest

from this_studio_b200 import batch, scenes, serve

from .helpers import rel_err


def test_tiles_do_not_overlap():
    rng = np.random.default_rng(0)
    boxes = []
    for _ in range(40):
        lo = rng.uniform(-1, 1, 3)
        boxes.append((lo, lo + rng.uniform(0.1, 0.5, 3)))
    gap = 0.05
    offs = batch.tile_offsets(boxes, gap)
    placed = [(np.asarray(lo) + o, np.asarray(hi) + o) for (lo, hi), o in zip(boxes, offs)]
    for i in range(len(placed)):
        for j in range(i + 1, len(placed)):
            a, b = placed[i], placed[j]
            sep = np.maximum(a[0] - b[1], b[0] - a[1])[:2].max()
            assert sep >= gap - 1e-12
    assert all(o[2] == 0 for o in offs)


def test_stream_is_seeded():
    a = serve.make_stream(20, seed=3)
    b = serve.make_stream(20, seed=3)
    assert [(r.kind, r.n, r.arrival) for r in a] == [(r.kind, r.n, r.arrival) for r in b]
    assert all(1000 <= r.n <= 200_000 for r in a)


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
def test_dem_member_same_alone_and_in_mix(gpu, prec, tol):
    x = scenes.dem_drop_poly(1500, seed=1)
    others = [scenes.dem_drop_poly(n, seed=s) for n, s in ((800, 2), (2500, 3), (1200, 4))]
    alone = scenes.build_dem(x, prec)
    alone.step(100)
    pa = alone.getBall()["position"]
    b = batch.DEMBatch(prec)
    b.members = [batch.Member(0, x), batch.Member(1, others[0]), batch.Member(2, others[1])]
    b.rebuild()
    b.step(45)
    # membership changes at a multiple of 5 steps: one leaves, one arrives
    b.capture()
    keep = {m.key: m for m in b.members}
    b.members = [keep[0], keep[2], batch.Member(3, others[2])]
    b.rebuild()
    b.step(55)
    b.capture()
    pm = b.members[0].state["position"]
    assert b.members[0].steps_done == 100
    e = rel_err(pm - x.position, pa - x.position)
    print(f"{prec}: DEM displacement alone vs in the mix {e:.2e}")
    assert e < tol


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
def test_sph_member_same_alone_and_in_mix(gpu, prec, tol):
    c0, dt = serve.stream_params(20000)
    x = scenes.sph_column(8000, c0, dt)
    others = [scenes.sph_column(n, c0, dt) for n in (3000, 12000)]
    alone = scenes.build_sph(x, prec)
    alone.step(60)
    pa = alone.getSPH()["position"]
    b = batch.SPHBatch(prec)
    b.members = [batch.Member(0, others[0]), batch.Member(1, x)]
    b.rebuild()
    b.step(25)
    b.capture()
    keep = {m.key: m for m in b.members}
    b.members = [keep[1], batch.Member(2, others[1])]
    b.rebuild()
    b.step(35)
    b.capture()
    pm = b.members[0].state["position"]
    e = rel_err(pm - x.fluid, pa - x.fluid)
    print(f"{prec}: SPH displacement alone vs in the mix {e:.2e}")
    assert e < tol


@pytest.mark.gpu
def test_server_completes_stream_and_matches_alone(gpu):
    reqs = serve.make_stream(10, seed=11, n_min=1000, n_max=8000, rate=400.0, steps=60)
    srv = serve.SceneServer(hbm_budget=2e9, chunk=20, precision="fp64", keep_states=True)
    m = srv.run(reqs)
    assert all(r.done is not None and r.final is not None for r in reqs)
    assert m["scene_step_latency_p99_ms"] >= m["scene_step_latency_p50_ms"] > 0
    c0, dt = srv.sph_c0, srv.sph_dt
    for r in reqs[:4]:
        sc = r.build(c0, dt)
        s = scenes.build_dem(sc, "fp64") if r.kind == "dem" else scenes.build_sph(sc, "fp64")
        s.step(r.steps)
        ref = s.getBall()["position"] if r.kind == "dem" else s.getSPH()["position"]
        base = sc.position if r.kind == "dem" else sc.fluid
        e = rel_err(r.final["position"] - base, ref - base)
        print(f"request {r.key} ({r.kind}, {r.np_} particles): served vs alone {e:.2e}")
        assert e < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_sph_assemble_matches_initialize(gpu, prec):
    """A scene assembled on the device from member records is the scene
    initialize() builds from the same particles: identical after 5 steps."""
    from this_studio_b200.solvers import SPHMember, WCSPHSolver

    c0, dt = serve.stream_params(20000)
    scs = [scenes.sph_column(n, c0, dt) for n in (3000, 5000)]
    offs = [np.zeros(3), np.array([1.5, 0.0, 0.0])]
    lo = np.min([np.asarray(sc.minb) + o for sc, o in zip(scs, offs)], axis=0)
    hi = np.max([np.asarray(sc.maxb) + o for sc, o in zip(scs, offs)], axis=0)
    a = WCSPHSolver()
    for sc, o in zip(scs, offs):
        a.addSPHs(sc.fluid + o, None, sc.sound_speed, sc.spacing, sc.density, sc.viscosity)
    for sc, o in zip(scs, offs):
        a.addDummies(sc.dummy + o, None, sc.sound_speed, sc.spacing, sc.density, sc.viscosity)
    a.initialize(lo, hi, scs[0].gravity, scs[0].dt, prec)
    recs = []
    for sc in scs:
        r = SPHMember()
        r.addSPHs(sc.fluid, None, sc.sound_speed, sc.spacing, sc.density, sc.viscosity)
        r.addDummies(sc.dummy, None, sc.sound_speed, sc.spacing, sc.density, sc.viscosity)
        recs.append(r.seal())
    assert recs[1].num() == scs[1].fluid.shape[0] and recs[1].num(True) == scs[1].dummy.shape[0]
    b = WCSPHSolver()
    b.assemble(recs, offs, lo, hi, scs[0].gravity, scs[0].dt, prec)
    np.testing.assert_array_equal(a.getDummy()["normal"], b.getDummy()["normal"])
    a.step(5)
    b.step(5)
    sa, sb = a.getSPH(), b.getSPH()
    for k in ("position", "velocity", "density", "pressure"):
        np.testing.assert_array_equal(sa[k], sb[k])


@pytest.mark.gpu
def test_dem_assemble_matches_host_build(gpu):
    """Balls placed on the device from member records give the scene that
    adding the same balls from the host gives: identical after 12 steps."""
    from this_studio_b200.solvers import DEMMember

    scs = [scenes.dem_drop_poly(n, seed=s) for n, s in ((900, 1), (1400, 2))]
    b = batch.DEMBatch("mixed")
    b.members = [batch.Member(k, sc) for k, sc in enumerate(scs)]
    prep = b.prepare(b.members)  # device assembly from member records
    # the same batch from host arrays: members carrying their initial state
    h = batch.DEMBatch("mixed")
    h.members = [batch.Member(k, sc, state={"position": sc.position.copy()}) for k, sc in enumerate(scs)]
    hprep = h.prepare(h.members)
    assert prep.ranges == hprep.ranges and prep.tri_ranges == hprep.tri_ranges
    prep.solver.step(12)
    hprep.solver.step(12)
    pa, pb = prep.solver.getBall(), hprep.solver.getBall()
    for k in ("position", "velocity", "angularVelocity"):
        np.testing.assert_array_equal(pa[k], pb[k])
    assert DEMMember is not None


def _sorted_bonds(bo, base=0):
    key = np.lexsort((bo["objectPointing"], bo["objectPointed"]))
    return {k: v[key] for k, v in bo.items()}


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
def test_dem_clumps_and_bonds_same_alone_and_in_mix(gpu, prec, tol):
    """Members with clumps and bonds (agglomerates bonded on their initial
    contacts, rigid 3-sphere clumps) keep their bodies across a membership
    change: balls, pebbles, clump states and bond states after 100 steps match
    the scene run alone."""
    x = scenes.dem_agglomerate_drop(1500, seed=1)
    y = scenes.dem_agglomerate_drop(2400, seed=2)
    rng = np.random.default_rng(0)
    for sc in (x, y):  # stress the bonds and spin the clumps from the first step
        sc.velocity = rng.normal(0.0, 0.05, sc.position.shape)
        for c in sc.clumps:
            c["angularVelocity"] = tuple(rng.normal(0.0, 20.0, 3))
    others = [scenes.dem_drop_poly(800, seed=3), scenes.dem_drop_poly(1200, seed=4),
              scenes.dem_agglomerate_drop(900, seed=5)]
    alone = {}
    for k, sc in ((0, x), (1, y)):
        s = scenes.build_dem(sc, prec)
        s.step(100)
        alone[k] = (s.getBall(), s.getClump(), s.getBondedInteraction())
    b = batch.DEMBatch(prec)
    b.members = [batch.Member(1, y), batch.Member(2, others[0]), batch.Member(0, x)]
    b.rebuild()
    b.step(45)
    keep = {m.key: m for m in b.members}
    # x and y continue at other indices; one leaves, two arrive
    b.members = [batch.Member(3, others[1]), keep[0], batch.Member(4, others[2]), keep[1]]
    b.rebuild()
    b.step(55)
    b.capture()
    got = {m.key: m for m in b.members}
    for k, sc in ((0, x), (1, y)):
        st = got[k].state
        assert got[k].steps_done == 100
        ball, cl, bo = alone[k]
        p0 = np.concatenate([sc.position] + [np.asarray(c["point"]) for c in sc.clumps])
        e_pos = rel_err(st["position"] - p0, ball["position"] - p0)
        e_clump = rel_err(st["clumps"]["position"] - np.array([c["centroid"] for c in sc.clumps]),
                          cl["position"] - np.array([c["centroid"] for c in sc.clumps]))
        e_q = np.abs(st["clumps"]["orientation"] - cl["orientation"]).max()
        mine, ref = _sorted_bonds(st["bonds"]), _sorted_bonds(bo)
        np.testing.assert_array_equal(mine["objectPointed"], ref["objectPointed"])
        np.testing.assert_array_equal(mine["objectPointing"], ref["objectPointing"])
        np.testing.assert_array_equal(mine["isBonded"], ref["isBonded"])
        e_fn = np.abs(mine["normalForce"] - ref["normalForce"]).max() / np.abs(ref["normalForce"]).max()
        print(f"{prec} member {k}: {len(sc.clumps)} clumps, {len(ref['isBonded'])} bonds; alone vs in the mix: "
              f"displacement {e_pos:.2e}, clump displacement {e_clump:.2e}, orientation {e_q:.2e}, "
              f"bond normal force {e_fn:.2e}")
        assert len(ref["isBonded"]) > 0 and len(sc.clumps) > 0
        assert e_pos < tol and e_clump < tol and e_q < tol
        assert e_fn < (1e-7 if prec == "fp64" else 1e-3)


@pytest.mark.gpu
def test_server_serves_bonded_and_clump_scenes(gpu):
    """The DEM batch of the server takes agglomerate / clump scenes beside
    plain drops; each result equals the scene run alone."""
    reqs = serve.make_stream(8, seed=21, n_min=1000, n_max=4000, rate=400.0, steps=40,
                             kinds=("dem", "dem_bonded", "sph"))
    assert any(r.kind == "dem_bonded" for r in reqs)
    srv = serve.SceneServer(hbm_budget=2e9, chunk=20, precision="fp64", keep_states=True)
    srv.run(reqs)
    c0, dt = srv.sph_c0, srv.sph_dt
    checked = 0
    for r in reqs:
        if r.kind != "dem_bonded":
            continue
        sc = r.build(c0, dt)
        s = scenes.build_dem(sc, "fp64")
        s.step(r.steps)
        ref = s.getBall()["position"]
        p0 = np.concatenate([sc.position] + [np.asarray(c["point"]) for c in sc.clumps])
        e = rel_err(r.final["position"] - p0, ref - p0)
        print(f"request {r.key} (dem_bonded, {r.np_} particles): served vs alone {e:.2e}")
        assert e < 1e-9
        checked += 1
    assert checked > 0
