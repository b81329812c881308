"""The autotuner (this_studio_b200/autotune.py) on the GPU: every cell size it
may choose gives the same pairs and, up to rounding, the same steps; the
tunings it returns build working batch scenes and a served stream."""
import numpy as np
import pytest

from this_studio_b200 import autotune, batch, scenes, serve

from .helpers import rel_err

pytestmark = pytest.mark.gpu


def _pair_set(a, b):
    lo, hi = np.minimum(a, b).astype(np.int64), np.maximum(a, b).astype(np.int64)
    return np.unique(lo * (1 << 32) + hi)


@pytest.mark.parametrize("factor", autotune.DEM_FACTORS[1:])
def test_dem_cell_factor_same_pairs_and_steps(gpu, factor):
    sc = scenes.dem_pack(n_side=12)
    a = scenes.build_dem(sc, "fp64")
    b = scenes.build_dem(sc, "fp64", configure=lambda s: s.setCellFactor(factor))
    for s in (a, b):
        s.step(23)
    pa, pb = a.getPairs(0), b.getPairs(0)
    np.testing.assert_array_equal(_pair_set(pa["objectPointed"], pa["objectPointing"]),
                                  _pair_set(pb["objectPointed"], pb["objectPointing"]))
    x0 = sc.position
    e = rel_err(b.getBall()["position"] - x0, a.getBall()["position"] - x0)
    print(f"DEM cell factor {factor}: {len(pa['objectPointed'])} pairs, displacement vs factor 1: {e:.2e}")
    assert e < 1e-10


@pytest.mark.parametrize("factor", autotune.SPH_FACTORS[1:])
def test_sph_cell_factor_same_pairs_and_steps(gpu, factor):
    sc = scenes.dam_break_reference()
    a = scenes.build_sph(sc, "fp64")
    b = scenes.build_sph(sc, "fp64", configure=lambda s: s.setCellFactor(factor))
    for s in (a, b):
        s.step(12)
        s.neighborSearch()
    for which in (0, 1):
        ia, ja = a.getPairs(which)
        ib, jb = b.getPairs(which)
        # rows come back in the reference's order whatever the grid
        np.testing.assert_array_equal(ia, ib)
        np.testing.assert_array_equal(ja, jb)
    x0 = sc.fluid
    e = rel_err(b.getSPH()["position"] - x0, a.getSPH()["position"] - x0)
    print(f"SPH cell factor {factor}: displacement vs factor 1: {e:.2e}")
    assert e < 1e-10


def test_tunings_build_batches_that_match_alone(gpu):
    dem = scenes.dem_drop_poly(3000, seed=7)
    td = autotune.tune_dem(dem, "fp64", steps=20, warmup=5)
    print("DEM tuning:", td.as_dict())
    assert td.cell_factor in autotune.DEM_FACTORS and min(td.reserve) >= 0
    c0, dt = serve.stream_params(20000)
    sph = scenes.sph_column(6000, c0, dt)
    ts = autotune.tune_sph(sph, "fp64", steps=10, warmup=4, trials=2)
    print("SPH tuning:", ts.as_dict())
    assert ts.cell_factor in autotune.SPH_FACTORS and ts.headroom >= 0.125 - 1e-12
    # a batch built with each tuning: its member equals the scene alone
    for kind, sc, t in (("dem", dem, td), ("sph", sph, ts)):
        alone = scenes.build_dem(sc, "fp64") if kind == "dem" else scenes.build_sph(sc, "fp64")
        alone.step(30)
        b = (batch.DEMBatch if kind == "dem" else batch.SPHBatch)("fp64", tuning=t)
        other = scenes.dem_drop_poly(1000, seed=8) if kind == "dem" else scenes.sph_column(2000, c0, dt)
        b.members = [batch.Member(0, other), batch.Member(1, sc)]
        b.rebuild()
        b.step(30)
        b.capture()
        x0 = sc.position if kind == "dem" else sc.fluid
        ref = alone.getBall()["position"] if kind == "dem" else alone.getSPH()["position"]
        e = rel_err(b.members[1].state["position"] - x0, ref - x0)
        print(f"{kind}: tuned batch member vs alone {e:.2e}")
        assert e < 1e-9


def test_server_with_autotune(gpu):
    reqs = serve.make_stream(6, seed=4, n_min=1000, n_max=6000, rate=400.0, steps=40)
    srv = serve.SceneServer(hbm_budget=2e9, chunk=20, precision="mixed", autotune=True)
    m = srv.run(reqs)
    print({k: (v["cell_factor"], v["ms_per_step"]) for k, v in m["tuning"].items()}, f"tune {m['tune_s']:.2f} s")
    assert all(r.done is not None for r in reqs)
    assert set(m["tuning"]) == {r.batch_kind for r in reqs}
