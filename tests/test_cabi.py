"""The C ABI: every declared entry point is exported, and argument / scene
errors come back as status codes (no GPU needed for these)."""
import ctypes
import os
import re

import numpy as np
import pytest

import this_studio_b200 as tsb
from this_studio_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    hdr = open(os.path.join(ROOT, "include", "demsph.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(demsph_\w+|buildHashStartEnd|buildPrefixSum|launchAdd\w+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = _declared()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding covers the same set
    assert set(names) == set(_lib.SIGNATURES)


def test_version_and_counter():
    assert b"sm_100a" in _lib.lib().demsph_version()
    assert tsb.kernel_launches() >= 0


def test_empty_scene_is_rejected():
    s = tsb.DEMSolver()
    with pytest.raises(tsb.DemsphError) as e:
        s.initialize((0, 0, 0), (1, 1, 1), (0, 0, -9.81), 1e-5)
    assert e.value.code == _lib.ERR_SCENE


def test_bad_ball_is_rejected():
    s = tsb.DEMSolver()
    s.setHertzianPair(0, 0, 1e7, 1e6, 0.8)
    s.addBalls([[0.5, 0.5, np.nan]], None, None, 0.01, 1000.0, 0)
    with pytest.raises(tsb.DemsphError) as e:
        s.initialize((0, 0, 0), (1, 1, 1), (0, 0, -9.81), 1e-5)
    assert e.value.code == _lib.ERR_SCENE
    s2 = tsb.DEMSolver()
    s2.addBalls([[0.5, 0.5, 0.5]], None, None, -0.01, 1000.0, 0)
    with pytest.raises(tsb.DemsphError):
        s2.initialize((0, 0, 0), (1, 1, 1), (0, 0, -9.81), 1e-5)


def test_bad_arguments():
    s = tsb.DEMSolver()
    s.addBalls([[0.5, 0.5, 0.5]], None, None, 0.01, 1000.0, 0)
    with pytest.raises(tsb.DemsphError) as e:
        s.initialize((0, 0, 0), (1, 1, 1), (0, 0, -9.81), -1.0)
    assert e.value.code == _lib.ERR_INVALID
    with pytest.raises(tsb.DemsphError) as e:
        s.step(1)
    assert e.value.code == _lib.ERR_NOT_READY
    with pytest.raises(tsb.DemsphError) as e:
        s.setMeshWallMotion(3, (0, 0, 0), (0, 0, 0))
    assert e.value.code == _lib.ERR_INVALID
    rc = _lib.lib().demsph_dem_step(None, 1)
    assert rc == _lib.ERR_INVALID
    sp = tsb.WCSPHSolver()
    with pytest.raises(tsb.DemsphError) as e:
        sp.initialize((0, 0, 0), (1, 1, 1), (0, 0, -9.81), 1e-5)
    assert e.value.code == _lib.ERR_SCENE


def test_cuda_failure_is_a_status_not_a_crash():
    import torch

    if torch.cuda.is_available():
        pytest.skip("needs a machine without a GPU")
    s = tsb.DEMSolver()
    s.setHertzianPair(0, 0, 1e7, 1e6, 0.8)
    s.addBalls([[0.5, 0.5, 0.5]], None, None, 0.01, 1000.0, 0)
    with pytest.raises(tsb.DemsphError) as e:
        s.initialize((0, 0, 0), (1, 1, 1), (0, 0, -9.81), 1e-5)
    assert e.value.code == _lib.ERR_CUDA
