"""The reference's own scene programs on this library.

* DEMSPH/elasticBounce.cpp, compiled unchanged against include/demsph_compat
  (oracle/Makefile.ref builds it, with the other three example mains, into
  oracle/_ref/scenes/ where the reference checkout is present): its 201 VTU
  frames against the reference's own frames (tests/golden/elastic_bounce.npz,
  one sphere on a 2-triangle wall, 20,000 steps).
* tests/cpp/beam_hook.cpp, a bonded cantilever written the way the
  reference's bondedParticleBeam.cpp is (addExternalForceTorque calling
  launchAddConstantForce / launchAddGlobalDampingForceTorque on getBall()'s
  arrays with a HostDeviceArray1D of its own, addInitialCondition bonding the
  initial contacts), compiled here against the same headers: its final state
  against the FP64 oracle.
"""
import os
import subprocess

import numpy as np
import pytest

from .golden.make_golden import read_vtu
from .helpers import oracle_dem, rel_err
from .test_gpu_dem import _beam

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
SCENES = os.path.join(ROOT, "oracle", "_ref", "scenes")


def test_reference_elastic_bounce_main(gpu, tmp_path):
    exe = os.path.join(SCENES, "elasticBounce")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/scenes not built (no reference checkout at build time)")
    r = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    fx = np.load(os.path.join(GOLDEN, "elastic_bounce.npz"))
    worst = 0.0
    for f in range(201):
        v = read_vtu(str(tmp_path / "elasticBounce" / ("ball_%04d.vtu" % f)), [("velocity", 3)])
        assert v["step"] == fx["step"][f]
        worst = max(worst, np.abs(v["position"][0] - fx["position"][f]).max(),
                    np.abs(v["velocity"][0] - fx["velocity"][f]).max())
    print(f"elasticBounce.cpp on this library (mixed precision): worst frame deviation {worst:.2e}")
    assert worst < 2e-5  # the frames carry 10 decimals; FP32 force laws


@pytest.mark.parametrize("prec", [0, 1])
def test_reference_style_hook_scene(gpu, oracle_lib, tmp_path, prec):
    exe = tmp_path / "beam_hook"
    cmd = ["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include", "demsph_compat"),
           "-I/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", "beam_hook.cpp"), "-o", str(exe),
           "-L" + os.path.join(ROOT, "this_studio_b200"), "-ldemsph_b200",
           "-Wl,-rpath," + os.path.join(ROOT, "this_studio_b200")]
    c = subprocess.run(cmd, capture_output=True, text=True)
    assert c.returncode == 0, c.stderr
    t_max = 0.05
    r = subprocess.run([str(exe), str(t_max), str(prec)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    lines = r.stdout.split("\n")
    calls = int([l for l in lines if l.startswith("hook_calls")][0].split()[1])
    pos = np.array([[float(x) for x in l.split()[1:]] for l in lines if l.startswith("pos ")])
    sc, f = _beam()
    steps = int(t_max / sc.dt) + 2  # solve's step count (DEMSolver.h:1988,1380)
    assert calls == 2 * steps
    o = oracle_dem(sc)
    o.set_constant_force(f, ramp=1.0)
    o.set_global_damping(0.1)
    o.step(steps)
    e = rel_err(pos - sc.position, o.balls()["pos"] - sc.position)
    print(f"hook scene ({'mixed' if prec else 'fp64'}), {steps} steps: displacement rel err {e:.2e} vs oracle")
    assert e < (1e-10 if prec == 0 else 1e-5)
