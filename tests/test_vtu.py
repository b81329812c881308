"""VTU frames and the reference scene generators, byte for byte against the
reference's own frame-0 files (sizes and SHA-256 in tests/golden/vtu_frame0.json,
made by tests/golden/make_golden.py from the reference's output folders).

Frame 0 is the initial state as the reference's solve() writes it after
initialisation, so the elasticBounce and iceCylinderInteraction frames check
the writer and the generators (hexagonal sheet, cylinder mesh) exactly; the
damBreak frame checks the SPH writer and the dam-break particle generation."""
import hashlib
import json
import os

import pytest

from this_studio_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "vtu_frame0.json")


def _same(path, key):
    ref = json.load(open(GOLDEN))[key]
    data = open(path, "rb").read()
    return len(data) == ref["bytes"] and hashlib.sha256(data).hexdigest() == ref["sha256"]


def test_elastic_bounce_frame0(tmp_path):
    s = scenes.build_dem(scenes.elastic_bounce(), "fp64", initialize=False)
    s.writeVTU(str(tmp_path), 0, what=1)
    assert _same(tmp_path / "ball_0000.vtu", "elasticBounce/ball_0000.vtu")


def test_ice_cylinder_generators_frame0(tmp_path):
    sc = scenes.ice_cylinder_reference()
    assert sc.position.shape == (11600, 3)
    assert sc.walls[0]["vertices"].shape == (37 * 36 + 2, 3) and len(sc.walls[0]["tri0"]) == 36 * 36 * 2 + 72
    s = scenes.build_dem(sc, "fp64", initialize=False)
    s.writeVTU(str(tmp_path), 0, what=1 | 2)
    assert _same(tmp_path / "ball_0000.vtu", "iceCylinderInteraction/ball_0000.vtu")
    assert _same(tmp_path / "triangleWall_0000.vtu", "iceCylinderInteraction/triangleWall_0000.vtu")


def test_water_level_bisection():
    # static flotation: submerged fraction (R + h)^2 (2R - h) / (4 R^3) = 0.9
    h = scenes.static_sphere_water_level(0.1, 900.0, 1000.0)
    R = 0.1
    assert (R + h) ** 2 * (2 * R - h) / (4 * R ** 3) == pytest.approx(0.9, rel=1e-12)
    assert scenes.static_sphere_water_level(0.1, 1100.0, 1000.0) == 0.1


def test_hex_pbc_snaps_periodic_axis():
    pbc = scenes.make_hex_pbc_2d((0, 0, 0), (1.0, 1.0, 0), 0.1, True, True)
    assert pbc.nx == 10 and pbc.ny == 12
    assert pbc.max[1] == pytest.approx(12 * 0.1 * 3 ** 0.5 / 2)
    assert pbc.shearX == 0.0  # even row count
    pts, _ = scenes.hex_point_cloud((0, 0, 0), (1.0, 1.0, 0), 0.1, True, True)
    assert pts.shape == (120, 3)


@pytest.mark.gpu
def test_dam_break_and_ice_cylinder_frame0_after_initialise(gpu, tmp_path):
    s = scenes.build_sph(scenes.dam_break_reference(), "fp64")
    s.writeVTU(str(tmp_path), 0, what=1)
    assert _same(tmp_path / "SPH_0000.vtu", "damBreak/SPH_0000.vtu")
    d = scenes.build_dem(scenes.ice_cylinder_reference(), "fp64")
    d.writeVTU(str(tmp_path), 0)
    assert _same(tmp_path / "ball_0000.vtu", "iceCylinderInteraction/ball_0000.vtu")
    assert _same(tmp_path / "triangleWall_0000.vtu", "iceCylinderInteraction/triangleWall_0000.vtu")
    assert _same(tmp_path / "ballTriangleInteraction_0000.vtu",
                 "iceCylinderInteraction/ballTriangleInteraction_0000.vtu")
    for f in ("ballInteraction_0000.vtu", "bondedInteraction_0000.vtu"):
        assert (tmp_path / f).stat().st_size > 0


@pytest.mark.gpu
def test_solve_writes_frames_on_the_reference_cadence(gpu, tmp_path):
    sc = scenes.elastic_bounce()
    s = scenes.build_dem(sc, "fp64", initialize=False)
    # 0.05 s at dt = 1e-4: numStep = 501, 5 frames -> every 100 steps
    s.solve(sc.minb, sc.maxb, sc.gravity, 1e-4, 0.05, numFrame=5, dir=str(tmp_path), precision="fp64")
    names = sorted(p.name for p in tmp_path.glob("ball_*.vtu"))
    assert names == ["ball_%04d.vtu" % k for k in range(6)]
    text = (tmp_path / "ball_0005.vtu").read_text()
    assert 'Name="STEP"  NumberOfTuples="1" format="ascii"> 500 <' in text
