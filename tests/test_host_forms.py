"""Host logic of the batched / served forms and the autotuner, without a GPU:
the tuner's margin rule and how a tuning configures a scene, the request
kinds' routing to batches, and the bonded agglomerate scene's geometry."""
import numpy as np

from this_studio_b200 import autotune, scenes, serve


def test_pick_keeps_default_within_margin():
    ms = {1.0: 1.00, 1.25: 0.97, 1.5: 1.10}
    assert autotune._pick(1.0, ms, 0.05) == 1.0  # 3% faster: noise
    ms[1.5] = 0.90
    assert autotune._pick(1.0, ms, 0.05) == 1.5  # 10% faster: taken
    assert autotune._pick(0, {0: 1.0, 1: 0.5}, 0.0) == 1


class _FakeSolver:
    def __init__(self):
        self.calls = []

    def __getattr__(self, name):
        return lambda *a: self.calls.append((name,) + a)


def test_tuning_configures_and_finishes_a_scene():
    t = autotune.Tuning("dem", cell_factor=1.25, reserve=(16, 12, 8))
    f = _FakeSolver()
    t.configure(f)
    t.finish(f)
    assert f.calls == [("setCellFactor", 1.25), ("reserve", 16, 12, 8)]
    t = autotune.Tuning("sph", cell_factor=1.0, list_shape=2, skin=0.02, headroom=0.3)
    f = _FakeSolver()
    t.configure(f)
    t.finish(f)
    assert f.calls == [("setCellFactor", 1.0), ("setListHeadroom", 0.3), ("setListShape", 2), ("setSkin", 0.02)]
    d = autotune.Tuning("dem", ms_per_step={1.0: 0.1}).as_dict()
    assert d["ms_per_step"] == {"1.0": 0.1}


def test_request_kinds_route_to_batches():
    reqs = serve.make_stream(30, seed=2, n_min=1000, n_max=3000, kinds=("dem", "dem_bonded", "sph"))
    assert {r.kind for r in reqs} == {"dem", "dem_bonded", "sph"}
    for r in reqs:
        assert r.batch_kind == ("sph" if r.kind == "sph" else "dem")


def test_agglomerate_scene_geometry():
    sc = scenes.dem_agglomerate_drop(1500, seed=1)
    r = sc.radius[0]
    assert sc.bond_initial_contacts and len(sc.clumps) > 0
    assert sc.num_moving == sc.position.shape[0] + 3 * len(sc.clumps)
    # within a 27-sphere agglomerate: face neighbours overlap slightly (a
    # contact of definite sign, inside one 2 r_max cell), diagonals are apart
    p = sc.position[:27]
    d = np.linalg.norm(p[:, None] - p[None], axis=2)[np.triu_indices(27, 1)]
    face = d[d < 2.2 * r]
    assert len(face) == 54
    assert np.all(face < 2 * r) and np.all(face > 1.99 * r)
    # agglomerates and clumps are far apart: no pair across bodies
    pts = np.concatenate([sc.position] + [np.asarray(c["point"]) for c in sc.clumps])
    body = np.concatenate([np.arange(sc.position.shape[0]) // 27,
                           np.repeat(10_000 + np.arange(len(sc.clumps)), 3)])
    for k in range(0, pts.shape[0], 97):
        dk = np.linalg.norm(pts - pts[k], axis=1)
        near = (dk < 2.2 * r) & (body != body[k])
        assert not near.any()
