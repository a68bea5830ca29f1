"""Generate tests/golden/ref_*.npz / ref_*.json from runs of the reference solver itself.

    python tests/golden/make_reference_golden.py [scene ...]      # default: every scene

Needs the reference checkout (Continuum Liquid, default /root/reference or $CLB_REFERENCE_ROOT)
and g++: the reference's main(config) runs unmodified on the host through oracle/reference_run.py
(its Python host code over the pyopencl stand-in, its OpenCL kernels compiled for the CPU by
oracle/ref_build.py). The scenes are defined in tests/golden/reference_scenes.py.

Small scenes (`reference_scenes.SMALL`) are stored as compressed .npz: the first, second and last
output frames whole and a digest of every frame, the first step's intermediates (per-cell counts and offsets, the sorted particles, the P2G grid
velocity and fluid fraction, the velocity entering the pressure solve, its right-hand side and the
pressure, the projected velocity, the particle velocity after G2P) and the voxelised masks.
Large scenes (`reference_scenes.LARGE`) are stored as .json digests of the same arrays
(`reference_scenes.digest`) with per-frame particle counts and coordinate sums; the collider mask of
the 128^3 scene is also stored whole (packed bits).
"""

from __future__ import annotations

import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

import reference_scenes as rs  # noqa: E402

from oracle import reference_run  # noqa: E402


def generate(name: str) -> Path:
    cfg = rs.scene(name)
    start = time.time()
    record = reference_run.run(cfg, rs.meshes(cfg), capture_steps=1)
    seconds = time.time() - start
    messages = [{k: v for k, v in m.items()} for m in record["messages"]]
    step = record["steps"][0]
    meta = {"scene": name, "config_digest": rs.config_digest(cfg), "reference_seconds": round(seconds, 1),
            "messages": messages}
    meta["frames"] = [{"count": int(len(f)), "digest": rs.digest(f),
                       "sum": [float(x) for x in f.astype(np.float64).sum(axis=0)]} for f in record["frames"]]
    if name in rs.SMALL:
        last = len(record["frames"]) - 1
        arrays = {f"frame_{i:03d}": record["frames"][i] for i in sorted({0, 1, last})}
        arrays.update({f"s1_{k}": v for k, v in step.items()})
        arrays.update({f"mask_{k}": v for k, v in record["masks"].items()})
        path = HERE / f"ref_{name}.npz"
        np.savez_compressed(path, meta=np.array(json.dumps(meta)), **arrays)
    else:
        meta["step1"] = {k: rs.digest(v) for k, v in step.items()}
        meta["masks"] = {k: rs.digest(v) for k, v in record["masks"].items()}
        path = HERE / f"ref_{name}.json"
        path.write_text(json.dumps(meta, indent=1))
        if "obstacle" in record["masks"] and record["masks"]["obstacle"].any():
            mask = record["masks"]["obstacle"]
            np.savez_compressed(HERE / f"ref_{name}_obstacle.npz", shape=np.array(mask.shape),
                                bits=np.packbits(mask.reshape(-1).astype(bool)))
    print(f"{name}: {len(record['frames'])} frames, {seconds:.1f} s -> {path.name}", flush=True)
    return path


if __name__ == "__main__":
    names = sys.argv[1:] or [*rs.SMALL, *rs.LARGE]
    for scene_name in names:
        generate(scene_name)
