"""Generate the golden fixtures of this directory from the CPU oracle (test infrastructure).

    python tests/golden/make_golden.py

Each fixture holds one seeded scene's inputs (particles, collider triangles and mask) and the oracle's
values after `steps` reference steps: the last step's per-cell counts and offsets, sorted positions,
P2G velocity and fluid fraction, pressure right-hand side and pressure, the projected grid velocity,
and the final particle state. The reference itself has no tests or golden vectors (its OpenCL
programs cannot run on this machine), so these fixtures pin the restatement: tests/test_golden.py
re-runs the oracle and the CUDA backend against them.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

CASES = {
    # name: (scene factory, FLIP/PIC blend, steps)
    "dam_break_16": (lambda scenes: scenes.dam_break(16, seed=3), 1.0, 2),
    "collider_pool_16": (lambda scenes: scenes.collider_pool(16, seed=4, subdivisions=2), 0.95, 2),
}
TRACE = ("counts", "offsets", "sorted_pos", "p2g_u", "p2g_ff", "rhs", "pressure", "u", "v", "w")


def generate(name: str):
    from continuum_liquid_b200 import scenes
    from oracle import oracle

    factory, flip, steps = CASES[name]
    s = factory(scenes)
    obstacle = np.zeros(s.grid_shape, np.uint8)
    triangles = np.zeros((0, 3, 3), np.float32)
    for tris in s.obstacles:
        obstacle = oracle.voxelise(tris, s.grid_shape, s.dx, s.origin, obstacle)
        triangles = np.concatenate([triangles, np.asarray(tris, np.float32)])
    pos, vel = scenes.seed_particles(s, obstacle)
    sim = oracle.OracleSim(s.grid_shape, s.dx, pos, vel, obstacle=obstacle, dt=s.dt, flip_ratio=flip,
                           gravity=s.gravity)
    for _ in range(steps):
        sim.step()
    out = {"grid_shape": np.asarray(s.grid_shape, np.int32), "dx": np.float64(s.dx), "dt": np.float64(s.dt),
           "gravity": np.asarray(s.gravity, np.float64), "flip_ratio": np.float64(flip), "steps": np.int32(steps),
           "origin": np.asarray(s.origin, np.float64), "triangles": triangles, "obstacle": obstacle,
           "in_pos": pos, "in_vel": vel, "out_pos": sim.pos, "out_vel": sim.vel}
    for key in TRACE:
        out[key] = sim.trace[key]
    return out


def main():
    for name in CASES:
        data = generate(name)
        path = HERE / f"{name}.npz"
        np.savez_compressed(path, **data)
        print(f"{path.name}: {path.stat().st_size / 1024:.0f} KiB, {len(data['in_pos'])} particles")


if __name__ == "__main__":
    main()
