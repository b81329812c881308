"""The reference's own CUDA kernels (built from its sources into
oracle/_ref by oracle/Makefile.ref) against this library, on the same GPU:
pair lists in the same order, forces and short trajectories, and the step
time of both on the benchmark workload."""
import time

import numpy as np
import pytest

from this_studio_b200 import scenes
from this_studio_b200.scenes import build_dem, build_sph

from .helpers import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    from oracle import ref_harness

    if not ref_harness.available():
        pytest.skip("oracle/_ref/libdemsph_ref.so not built (make -f oracle/Makefile.ref)")
    return ref_harness


def test_sph_pairs_and_trajectory_match_reference_kernels(gpu, ref):
    import torch

    sc = scenes.dam_break_reference()
    r = ref.RefSPH(sc, torch)
    g = build_sph(sc, "fp64")
    assert rel_err(g.getDummy()["normal"], r.state()["dummy_normal"]) < 1e-13
    a, b = g.getPairs(2)
    ra, rb = r.pairs(2)
    np.testing.assert_array_equal(a, ra)
    np.testing.assert_array_equal(b, rb)
    r.neighbor_search()
    g.neighborSearch()
    for which in (0, 1):
        a, b = g.getPairs(which)
        ra, rb = r.pairs(which)
        np.testing.assert_array_equal(a, ra)
        np.testing.assert_array_equal(b, rb)
    r.step(30)
    g.step(30)
    s, rs = g.getSPH(), r.state()
    e = rel_err(s["position"] - sc.fluid, rs["pos"] - sc.fluid)
    print(f"30 steps vs reference kernels: displacement rel err {e:.2e}")
    assert e < 1e-10
    assert rel_err(s["density"] - 1000.0, rs["rho"] - 1000.0) < 1e-9
    assert rel_err(s["acceleration"], rs["acc"]) < 1e-9


def test_dem_pairs_and_forces_match_reference_kernels(gpu, ref):
    import torch

    sc = scenes.dem_pack(n_side=12)
    r = ref.RefDEMPairs(sc, torch)
    r.neighbor_search()
    g = build_dem(sc, "fp64")
    ra, rb = r.pairs()
    pg = g.getPairs(0)
    assert len(ra) > 3000
    np.testing.assert_array_equal(pg["objectPointed"], ra)
    np.testing.assert_array_equal(pg["objectPointing"], rb)
    fr, tr = r.forces(0.5 * sc.dt)
    g.evalForces(0.5 * sc.dt)
    b = g.getBall()
    ef, et = rel_err(b["force"], fr), rel_err(b["torque"], tr)
    print(f"DEM forces vs reference kernels: force {ef:.2e} torque {et:.2e}")
    assert ef < 1e-12 and et < 1e-12
    g2 = build_dem(sc, "mixed")
    g2.evalForces(0.5 * sc.dt)
    b2 = g2.getBall()
    print(f"mixed precision vs reference kernels: force {rel_err(b2['force'], fr):.2e}")
    assert rel_err(b2["force"], fr) < 1e-5


def test_step_time_against_reference_kernels(gpu, ref):
    """Both on the benchmark workload (128,000 fluid, 150,216 dummies)."""
    import torch

    sc = scenes.sph_dam_break()
    r = ref.RefSPH(sc, torch)
    r.step(3)
    torch.cuda.synchronize()
    n = 20
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    r.step(n)
    e1.record()
    e1.synchronize()
    ref_ms = e0.elapsed_time(e1) / n
    out = {}
    for prec in ("fp64", "mixed"):
        g = build_sph(sc, prec)
        g.step(3)
        torch.cuda.synchronize()
        e0.record()
        g.step(n)
        e1.record()
        e1.synchronize()
        out[prec] = e0.elapsed_time(e1) / n
    nf = sc.fluid.shape[0]
    print(f"reference CUDA build: {ref_ms:.3f} ms/step = {nf / ref_ms * 1e3:.3e} particle-steps/s; "
          f"this library fp64 {out['fp64']:.3f} ms/step ({ref_ms / out['fp64']:.1f}x), "
          f"mixed {out['mixed']:.3f} ms/step ({ref_ms / out['mixed']:.1f}x)")
    assert out["fp64"] < ref_ms
