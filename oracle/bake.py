"""ORACLE -- test infrastructure only; never imported by the product package.

A whole bake restated on the CPU: `Solver/Kernel/solver.py:22-531` (what `Solver/General/main.py`
main(config) runs) over the oracle's kernels (oracle.py) and host sources (sources.py). It reads the
same config keys, voxelises every source and obstacle mesh (`voxelise_mesh.py:111-163`), seeds the
initial particles and applies inflows and outflows before every step with `default_rng(0)`, steps
with the reference's fixed gravity (0, 0, -9.81), pure FLIP and `settings.iterations` W-cycles, and
records the particle positions of every output frame.
"""

from __future__ import annotations

import numpy as np

from . import oracle
from . import sources as host_sources

FIELD_DTYPE = np.float32


def world_triangles(entry) -> np.ndarray:
    """voxelise_mesh.py:103-109 for an entry that carries its triangles: tri @ M[:3,:3]^T + M[:3,3]."""
    triangles = np.ascontiguousarray(entry["triangles"], dtype=np.float32).reshape(-1, 3, 3)
    matrix = np.asarray(entry.get("matrix_world", np.eye(4)), dtype=np.float32)
    flat = triangles.reshape(-1, 3)
    world = flat @ matrix[:3, :3].T + matrix[:3, 3]
    return np.ascontiguousarray(world.reshape(-1, 3, 3), dtype=np.float32)


def voxelise_entries(entries, grid_shape, delta, origin) -> np.ndarray:
    """voxelise_mesh.py:111-135: one zeroed mask, every entry's mesh OR-ed in."""
    mask = np.zeros(grid_shape, np.uint8)
    for entry in entries or ():
        tris = world_triangles(entry)
        if tris.size:
            mask = oracle.voxelise(tris, grid_shape, delta, origin, mask)
    return mask


def bake(config: dict, max_frames: int | None = None) -> dict:
    """Runs the bake; returns {"frames": [(N,3) float32], "steps": [trace of the first step],
    "masks": {...}, "counts": [particles per frame]}."""
    simulation = config.get("simulation") or {}
    settings = simulation.get("settings") or {}
    domain = simulation["domain"]
    size = domain["size"]
    physics = simulation["physics"]
    start_frame = int(settings.get("start_frame", 1))
    end_frame = int(settings.get("end_frame", 250))
    fps = int(settings.get("fps", 24))
    steps_per_frame = max(0, int(settings.get("substeps", 1))) + 1
    total_frames = max(0, end_frame - start_frame)
    if max_frames is not None:
        total_frames = min(total_frames, max_frames)
    dt = 1.0 / (fps * steps_per_frame)
    delta = float(domain["resolution"])
    grid_shape = (int(float(size["x"]) / delta), int(float(size["y"]) / delta), int(float(size["z"]) / delta))
    origin = (-0.5 * float(size["x"]), -0.5 * float(size["y"]), 0.0)

    masks = {}
    source_list = []
    for i, source in enumerate(simulation.get("sources") or ()):
        mask = voxelise_entries(source.get("geometry_inputs"), grid_shape, delta, origin)
        masks[f"source{i}"] = mask
        entry = {k: v for k, v in source.items() if k != "geometry_inputs"}
        entry["mask"] = mask.astype(np.bool_)
        source_list.append(entry)
    obstacle_entries = [e for o in simulation.get("obstacles") or () for e in o.get("geometry_inputs") or ()]
    obstacle = voxelise_entries(obstacle_entries, grid_shape, delta, origin)
    masks["obstacle"] = obstacle
    obstacle_bool = obstacle.astype(np.bool_)

    rng = np.random.default_rng(0)
    pos = np.empty((0, 3), dtype=FIELD_DTYPE)
    vel = np.empty((0, 3), dtype=FIELD_DTYPE)
    pos, vel = host_sources.apply_sources(pos, vel, source_list, obstacle_bool, delta, rng, initial=True)
    sim = oracle.OracleSim(grid_shape, delta, pos, vel, obstacle=obstacle, dt=dt, flip_ratio=1.0,
                           gravity=(0.0, 0.0, -9.81), rho=float(physics["water"]["density"]),
                           nu=float(physics["water"]["viscosity"]), ppc=8, min_size=8,
                           num_vcycles=max(1, int(settings.get("iterations", 1))))
    frames = [sim.pos.copy()]
    steps = []
    dynamic = any(s.get("type") in {"INFLOW", "OUTFLOW"} for s in source_list)
    for solver_step in range(total_frames * steps_per_frame):
        substep_index = solver_step % steps_per_frame
        if dynamic:
            sim.pos, sim.vel = host_sources.apply_sources(sim.pos, sim.vel, source_list, obstacle_bool, delta, rng)
        if len(sim.pos) == 0:
            if substep_index == steps_per_frame - 1:
                frames.append(sim.pos.copy())
            continue
        sim.step()
        if not steps:
            steps.append(dict(sim.trace))
        if substep_index == steps_per_frame - 1:
            frames.append(sim.pos.copy())
    return {"frames": frames, "steps": steps, "masks": masks, "grid_shape": grid_shape, "delta": delta}
