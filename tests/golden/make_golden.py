"""Extract golden fixtures from the reference's own output frames.

The reference (kaiqideng/this_studio, DEMSPH/) ships ASCII VTU frames written
by its FP64 CUDA build.  This script reads them from a checkout of the
reference and writes small fixtures next to it:

* ``elastic_bounce.npz`` -- all 201 frames of DEMSPH/elasticBounce/ball_*.vtu
  (one sphere, linear spring, 2-triangle wall; scene in DEMSPH/elasticBounce.cpp):
  time, step, position, velocity.
* ``dam_break_f1.npz`` -- frame 1 (step 670) of DEMSPH/damBreak/SPH_*.vtu for
  every 16th fluid particle (scene in DEMSPH/damBreak.cpp): index, position,
  velocity, density, pressure; plus frame-0 positions of the same subset.
* ``vtu_frame0.json`` -- size and SHA-256 of the reference's frame-0 VTU files
  of the elasticBounce, damBreak and iceCylinderInteraction scenes (the
  initial state as the reference writes it), to check the VTU writer and the
  scene generators byte for byte.

Usage:  python tests/golden/make_golden.py /path/to/reference
"""
import os
import re
import sys

import numpy as np


def read_vtu(path, fields):
    text = open(path).read()
    out = {}
    out["time"] = float(re.search(r'Name="TIME"[^>]*>\s*([-\d.eE+]+)', text).group(1))
    out["step"] = int(re.search(r'Name="STEP"[^>]*>\s*(\d+)', text).group(1))
    pts = re.search(r"<Points>\s*<DataArray[^>]*>(.*?)</DataArray>", text, re.S).group(1)
    out["position"] = np.array(pts.split(), float).reshape(-1, 3)
    for name, ncomp in fields:
        m = re.search(r'Name="%s"[^>]*>(.*?)</DataArray>' % name, text, re.S)
        a = np.array(m.group(1).split(), float)
        out[name] = a.reshape(-1, ncomp) if ncomp > 1 else a
    return out


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    eb = os.path.join(ref, "DEMSPH", "elasticBounce")
    frames = [read_vtu(os.path.join(eb, "ball_%04d.vtu" % f), [("velocity", 3)]) for f in range(201)]
    np.savez_compressed(
        os.path.join(here, "elastic_bounce.npz"),
        time=np.array([f["time"] for f in frames]),
        step=np.array([f["step"] for f in frames], np.int64),
        position=np.array([f["position"][0] for f in frames]),
        velocity=np.array([f["velocity"][0] for f in frames]),
    )
    db = os.path.join(ref, "DEMSPH", "damBreak")
    f0 = read_vtu(os.path.join(db, "SPH_0000.vtu"), [])
    f1 = read_vtu(os.path.join(db, "SPH_0001.vtu"), [("velocity", 3), ("density", 1), ("pressure", 1)])
    idx = np.arange(0, f1["position"].shape[0], 16)
    np.savez_compressed(
        os.path.join(here, "dam_break_f1.npz"),
        num_fluid=np.int64(f1["position"].shape[0]),
        step=np.int64(f1["step"]),
        time=np.float64(f1["time"]),
        index=idx.astype(np.int64),
        position0=f0["position"][idx],
        position=f1["position"][idx],
        velocity=f1["velocity"][idx],
        density=f1["density"][idx],
        pressure=f1["pressure"][idx],
    )
    import hashlib
    import json

    frame0 = {}
    for rel in ("elasticBounce/ball_0000.vtu", "damBreak/SPH_0000.vtu", "iceCylinderInteraction/ball_0000.vtu",
                "iceCylinderInteraction/triangleWall_0000.vtu",
                "iceCylinderInteraction/ballTriangleInteraction_0000.vtu"):
        data = open(os.path.join(ref, "DEMSPH", rel), "rb").read()
        frame0[rel] = {"bytes": len(data), "sha256": hashlib.sha256(data).hexdigest()}
    with open(os.path.join(here, "vtu_frame0.json"), "w") as f:
        json.dump(frame0, f, indent=1)
    print("wrote fixtures to", here)


if __name__ == "__main__":
    # the reference checkout: first argument, else DEMSPH_REFERENCE, else
    # where it is mounted in the build container
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DEMSPH_REFERENCE", "/root/reference"))
