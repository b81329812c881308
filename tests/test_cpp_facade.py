"""The C++ facade (include/demsph/solvers.hpp) compiles against the C ABI,
links against libdemsph_b200.so and reports failures as exceptions."""
import os
import subprocess

import pytest

from this_studio_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <demsph/solvers.hpp>
#include <cstdio>
int main() {
    demsph::DEMSolver test(0);
    test.setLinearPair(0, 0, 1e3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0);
    try {  // empty scene: rejected before any device work
        test.initialize(make_double3(-1, -1, -1), make_double3(1, 1, 1), make_double3(0, 0, -9.81), 1e-4);
        return 2;
    } catch (const demsph::Error& e) {
        std::printf("code %d\n", e.code);
    }
    test.addBall(make_double3(0, 0, 0), make_double3(0, 0, 0), make_double3(0, 0, 0), 0.01, 2000, 0);
    demsph::WCSPHSolver sph(0);
    sph.addSPH(make_double3(0, 0, 0), make_double3(0, 0, 0), 20.0, 0.01, 1000.0, 1e-3);
    std::printf("ok %ld\n", demsph::solveSteps(1e-4, 2.0));
    return 0;
}
"""


def test_facade_builds_and_runs(tmp_path):
    src = tmp_path / "scene.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "scene"
    libdir = os.path.dirname(_lib.LIB_PATH)
    cmd = ["g++", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include", str(src),
           "-o", str(exe), _lib.LIB_PATH, "-Wl,-rpath," + libdir]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "code 2" in out.stdout  # DEMSPH_ERR_SCENE
    assert "ok 20001" in out.stdout or "ok 20002" in out.stdout
