"""Named synthetic workloads, run for a few steps (for profiling a kernel on
a given scene):

    python -m this_studio_b200.workloads sph_dam_break_1m --steps 3

sph_dam_break_128k  WCSPH dam break, 40 x 40 x 80 fluid at dx = 0.01 (128,000)
sph_dam_break_1m    the same tank at dx = 0.005: 80 x 80 x 160 fluid (1,024,000)
dem_drop_4096       4,096 Hertz-Mindlin spheres dropped onto a plane
dem_drop_1m         about 10^6 polydisperse spheres dropped onto a plane
bonded_beam_clumps  a 20 x 20 x 400 bonded beam of r = 1 mm spheres (about 464k
                    parallel bonds, one end clamped, random tip load) beside
                    20,000 three-sphere clumps, dt = 1e-7
ice_sheet_coupled   about 1M bonded r = 2 mm spheres (ice, E = 9e9) moving into a
                    20,000-triangle cylinder, floating on 2M WCSPH particles at
                    dx = 4 mm, coupled particle by particle
coupled_tank_200k   eight DEM balls (r = 6 dx) in a 64 x 64 x 48 tank of water
                    at dx = 0.01 (about 190,000 fluid particles), coupled
                    particle by particle, two DEM substeps per fluid step
"""
from __future__ import annotations

import argparse

from . import scenes


COUPLED_BALLS = ((0.25, 0.25, 0.35, 6.0, 2500.0), (0.75, 0.25, 0.35, 6.0, 500.0), (0.25, 0.75, 0.35, 6.0, 1200.0),
                 (0.75, 0.75, 0.35, 6.0, 800.0), (0.25, 0.25, 0.75, 6.0, 2500.0), (0.75, 0.25, 0.75, 6.0, 500.0),
                 (0.25, 0.75, 0.75, 6.0, 1200.0), (0.75, 0.75, 0.75, 6.0, 800.0))


def coupled_tank_scene():
    return scenes.balls_in_tank(nx=64, ny=64, depth=48, balls=COUPLED_BALLS, dem_substeps=2)


def build(name, precision="mixed"):
    if name == "coupled_tank_200k":
        return scenes.build_coupled(coupled_tank_scene(), precision)[2]
    if name == "bonded_beam_clumps":
        return scenes.build_dem(scenes.bonded_beam_clumps(), precision)
    if name == "ice_sheet_coupled":
        return scenes.build_coupled(scenes.ice_sheet_on_water(), precision)[2]
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
    ap.add_argument("--flush-l2", action="store_true",
                    help="one step at a time with a 256 MB write between steps (as bench.py times them)")
    a = ap.parse_args()
    s = build(a.name, a.precision)
    if a.name.startswith("coupled") or a.name.startswith("ice_sheet"):
        if a.no_graphs:
            s.sph.setGraphs(False)
            s.dem.setGraphs(False)
        s.step(a.steps, 2 if a.name.startswith("coupled") else 1)
        s.sph.stepIndex()
    else:
        if a.no_graphs:
            s.setGraphs(False)
        if a.flush_l2:
            import torch

            flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
            for _ in range(a.steps):
                flush.zero_()
                s.step(1)
        else:
            s.step(a.steps)
        s.stepIndex()
    print(f"{a.name}: {a.steps} steps done")


if __name__ == "__main__":
    main()
