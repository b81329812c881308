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


class _FakeBatch:
    """The batch interface without a device: a step advances the members'
    step counts; commits are recorded with the members' total bytes."""

    def __init__(self, kind, sizes, max_members, shared):
        self.kind, self.sizes, self.max_members, self.shared = kind, sizes, max_members, shared
        self.members = []
        self.timing = {"initialize_s": 0.0, "carry_s": 0.0, "rebuilds": 0}

    def prepare(self, members):
        assert 0 < len(members) <= self.max_members
        assert all(self.sizes[m.key][0] == self.kind for m in members)
        return list(members)

    def commit(self, prep):
        self.members = prep
        self.timing["rebuilds"] += 1
        self.shared[self.kind] = sum(self.sizes[m.key][1] for m in prep)
        self.shared["peak"] = max(self.shared["peak"], self.shared.get("dem", 0) + self.shared.get("sph", 0))

    def step(self, n):
        import time

        for m in self.members:
            m.steps_done += n
        time.sleep(0.0005)

    def capture(self, keys=None):
        pass

    def clear(self):
        self.members = []
        self.shared[self.kind] = 0


def test_server_schedules_every_request_within_budget():
    """The served form's scheduling on fake batches: every request runs its
    steps to completion after it arrived, is admitted no earlier than its
    arrival, batches hold one kind and at most max_members, and the members
    committed at any time fit the HBM budget (every request here fits it alone)."""
    c0, dt = serve.stream_params(3000)
    reqs = serve.make_stream(40, seed=3, n_min=500, n_max=3000, rate=2000.0, steps=200)
    for r in reqs:
        r.build(c0, dt)
    sizes = {r.key: (r.batch_kind, r.bytes()) for r in reqs}
    budget = 4 * max(b for _, b in sizes.values())
    shared = {"peak": 0}
    fakes = {k: _FakeBatch(k, sizes, 6, shared) for k in ("dem", "sph")}
    srv = serve.SceneServer(hbm_budget=budget, chunk=50, max_members=6, sph_c0=c0, sph_dt=dt, batches=fakes)
    m = srv.run(reqs)
    assert all(r.done is not None and r.admitted is not None for r in reqs)
    assert all(r.admitted >= r.arrival - 1e-9 and r.done >= r.admitted for r in reqs)
    assert shared["peak"] <= budget
    assert m["scenes"] == 40 and m["particle_steps"] == sum(r.np_ * r.steps for r in reqs)
    for k in ("dem", "sph"):
        pk = m["per_kind"][k]
        assert pk["chunks"] >= 4 and pk["rebuilds"] >= 1
        assert {"busy_s", "prepare_wait_s", "idle_s", "commit_s"} <= set(pk)
