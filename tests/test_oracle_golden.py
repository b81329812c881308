"""The oracle against the reference's own output frames (CPU only).

The reference wrote these frames with its FP64 CUDA build; the fixtures were
extracted by tests/golden/make_golden.py.  Agreement here pins the oracle that
every GPU parity test is checked against.
"""
import os

import numpy as np
import pytest

from this_studio_b200 import scenes

from .helpers import oracle_dem, oracle_sph

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_elastic_bounce_all_frames(oracle_lib):
    fx = np.load(os.path.join(GOLDEN, "elastic_bounce.npz"))
    o = oracle_dem(scenes.elastic_bounce())
    worst = 0.0
    for f in range(1, 201):
        o.step(100)
        assert o.step_index == fx["step"][f]
        b = o.balls()
        worst = max(worst, np.abs(b["pos"][0] - fx["position"][f]).max(), np.abs(b["vel"][0] - fx["velocity"][f]).max())
    # frames carry 10 decimals; FP64 CPU vs FP64 GPU rounding stays below that
    assert worst < 1e-9, worst


@pytest.mark.slow
def test_dam_break_frame1(oracle_lib):
    fx = np.load(os.path.join(GOLDEN, "dam_break_f1.npz"))
    sc = scenes.dam_break_reference()
    assert sc.fluid.shape[0] == int(fx["num_fluid"])
    np.testing.assert_allclose(sc.fluid[fx["index"]], fx["position0"], atol=1e-10)
    o = oracle_sph(sc)
    o.step(int(fx["step"]))
    s = o.state()
    idx = fx["index"]
    # The flow amplifies last-bit differences (CPU 1/sqrt vs GPU rsqrt, FMA);
    # bounds are ~2x the worst deviation seen over all 18,081 particles.
    assert np.abs(s["pos"][idx] - fx["position"]).max() < 2e-7
    assert np.abs(s["vel"][idx] - fx["velocity"]).max() < 1e-5
    assert np.abs(s["rho"][idx] - fx["density"]).max() < 5e-5
    assert np.abs(s["p"][idx] - fx["pressure"]).max() < 2e-2
    assert np.median(np.abs(s["pos"][idx] - fx["position"])) < 2e-9


def _brute_pairs(p, r, im, clump=None):
    n = p.shape[0]
    out = set()
    for a in range(n):
        d = p[a] - p[a + 1:]
        cut = 1.1 * (r[a] + r[a + 1:])
        ok = (cut * cut - np.einsum("ij,ij->i", d, d)) >= 0
        for k in np.flatnonzero(ok):
            b = a + 1 + k
            if im[a] == 0 and im[b] == 0:
                continue
            out.add((a, b))
    return out


def test_oracle_pairs_vs_brute_force(oracle_lib):
    sc = scenes.dem_pack(n_side=6)
    o = oracle_dem(sc)
    pr = o.pairs(0)
    got = set(zip(pr["a"].tolist(), pr["b"].tolist()))
    im = np.ones(sc.position.shape[0])
    brute = _brute_pairs(sc.position, sc.radius, im)
    assert got <= brute
    # every pair closer than one cell (2 r_max) is inside the 27-cell stencil
    d = np.linalg.norm(sc.position[[a for a, _ in brute]] - sc.position[[b for _, b in brute]], axis=1)
    near = {pq for pq, dd in zip(brute, d) if dd < 2 * sc.radius.max()}
    assert near <= got
    # active contacts (overlap > 0) are all found
    assert all((a, b) in got for (a, b), dd in zip(brute, d) if dd < 2 * sc.radius[0])


def test_oracle_internal_forces_balance(oracle_lib):
    sc = scenes.dem_pack(n_side=6)
    o = oracle_dem(sc)
    o.step(3)
    o.eval_forces(0.5 * sc.dt)
    f = o.balls()["force"]
    assert np.abs(f.sum(0)).max() < 1e-12 * np.abs(f).sum()
