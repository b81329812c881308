"""The reference's external-force hook on the GPU: a callback in the style of
DEMSolver::addExternalForceTorque (DEMSolver.h:1372) that calls the
reference-signature launchers (launchAddConstantForce,
launchAddGlobalDampingForceTorque, launchAddBuoyancyDrag; externalForceTorque.h)
on the ball arrays in the reference's layout gives the same trajectory as the
same forces configured on the scene, and as the FP64 oracle."""
import ctypes as C

import numpy as np
import pytest

from this_studio_b200 import _lib, scenes
from this_studio_b200.scenes import build_dem

from .helpers import oracle_dem, rel_err
from .test_gpu_dem import _beam

pytestmark = pytest.mark.gpu


def _launchers():
    return _lib.lib()


def test_hook_callback_matches_configured_forces_and_oracle(gpu, oracle_lib):
    import torch

    sc, f = _beam()
    n = sc.position.shape[0]
    # the configured form
    a = build_dem(sc, "fp64")
    a.setConstantForce(f, rampTime=1.0)
    a.setGlobalDamping(0.1)
    # the hook form, written as bondedParticleBeam.cpp:17-42 writes it
    b = build_dem(sc, "fp64")
    fe = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    calls = []

    def hook(iStep, time):
        c = min(time, 1.0)
        fe.copy_(torch.from_numpy(f * c))
        arr = b.hookArrays()
        L = _launchers()
        L.launchAddConstantForce(arr.force, C.c_void_p(fe.data_ptr()), n, 0, 0, None)
        L.launchAddGlobalDampingForceTorque(arr.force, arr.torque, arr.velocity, arr.angularVelocity, 0.1, n, 0, 0,
                                            None)
        calls.append((iStep, time))

    b.setExternalHook(hook)
    steps = 300
    a.step(steps)
    b.step(steps)
    assert len(calls) == 2 * steps
    dt = sc.dt
    assert calls[0][0] == 1 and abs(calls[0][1] - 0.5 * dt) < 1e-18
    assert calls[-1][0] == steps and abs(calls[-1][1] - steps * dt) < 1e-12
    pa, pb = a.getBall(), b.getBall()
    e = rel_err(pb["position"] - sc.position, pa["position"] - sc.position)
    print(f"hook vs configured forces after {steps} steps: displacement rel err {e:.2e}")
    assert e < 1e-12
    assert rel_err(b.getBondedInteraction()["normalForce"], a.getBondedInteraction()["normalForce"]) < 1e-12
    o = oracle_dem(sc)
    o.set_constant_force(f, ramp=1.0)
    o.set_global_damping(0.1)
    o.step(steps)
    eo = rel_err(pb["position"] - sc.position, o.balls()["pos"] - sc.position)
    print(f"hook vs oracle: {eo:.2e}")
    assert eo < 1e-10
    # removing the hook from inside the callback: the next steps run without it
    removed = []

    def once(iStep, time):
        removed.append(iStep)
        b.setExternalHook(None)

    b.setExternalHook(once)
    b.step(3)
    assert removed == [steps + 1]


def test_buoyancy_launcher_in_a_hook(gpu, oracle_lib):
    import torch

    sc = scenes.dem_drop(n_side=5, plane_gap=0.002)
    lvl = float(sc.position[:, 2].mean())
    g3, u3 = (0.0, 0.0, -9.81), (-0.4, 0.0, 0.0)
    b = build_dem(sc, "fp64")
    n = sc.position.shape[0]

    def hook(iStep, time):
        arr = b.hookArrays()
        _launchers().launchAddBuoyancyDrag(arr.force, arr.position, arr.velocity, arr.radius, arr.inverseMass,
                                           1000.0, 0.1, _lib.Double3(*g3), _lib.Double3(*u3), lvl, n, 0, 0, None)

    b.setExternalHook(hook)
    b.step(200)
    sc.buoyancy = (1000.0, 0.1, g3, u3, lvl)
    o = oracle_dem(sc)
    o.step(200)
    e = rel_err(b.getBall()["velocity"], o.balls()["vel"])
    print(f"buoyancy through the reference launcher in a hook: velocity rel err {e:.2e}")
    assert e < 1e-9
    torch.cuda.synchronize()


def test_external_flag_applies_configured_forces(gpu):
    sc, f = _beam()
    g = build_dem(sc, "fp64")
    g.setConstantForce(f)
    g.evalForces(0.5 * sc.dt)
    f0 = g.getBall()["force"]
    g.evalForces(0.5 * sc.dt, external=True)
    f1 = g.getBall()["force"]
    assert np.allclose(f1 - f0, f, rtol=0, atol=1e-9)
