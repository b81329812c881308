"""Named synthetic workloads, run for a few steps (for profiling a kernel on
a given scene):

    python -m this_studio_b200.workloads sph_dam_break_1m --steps 3

sph_dam_break_128k  WCSPH dam break, 40 x 40 x 80 fluid at dx = 0.01 (128,000)
sph_dam_break_1m    the same tank at dx = 0.005: 80 x 80 x 160 fluid (1,024,000)
dem_drop_4096       4,096 Hertz-Mindlin spheres dropped onto a plane
dem_drop_1m         about 10^6 polydisperse spheres dropped onto a plane
"""
from __future__ import annotations

import argparse

from . import scenes


def build(name, precision="mixed"):
    if name == "sph_dam_break_128k":
        return scenes.build_sph(scenes.sph_dam_break(), precision)
    if name == "sph_dam_break_1m":
        return scenes.build_sph(scenes.sph_dam_break(nx=80, ny=80, nz=160, dx=0.005), precision)
    if name == "dem_drop_4096":
        return scenes.build_dem(scenes.dem_drop(), precision)
    if name == "dem_drop_1m":
        return scenes.build_dem(scenes.dem_drop_poly(1_000_000, seed=3), precision)
    raise ValueError(f"unknown workload {name}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("name")
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--no-graphs", action="store_true", help="launch every kernel directly")
    a = ap.parse_args()
    s = build(a.name, a.precision)
    if a.no_graphs:
        s.setGraphs(False)
    s.step(a.steps)
    s.stepIndex()
    print(f"{a.name}: {a.steps} steps done")


if __name__ == "__main__":
    main()
