"""Bake configurations that the reference solver itself was run on (test infrastructure).

Each scene is an add-on config for `main(config)` (the schema of `Internal/Core/export_config.py`,
as `Solver/Kernel/solver.py:22-240` reads it) that both solvers accept unchanged: every geometry
entry carries a `mesh_file` name, which the reference run resolves to the entry's triangles (USD
loading is bypassed, see oracle/reference_run.py), and the same world-space `triangles`, which this
backend reads directly. The domain is the unit cube with the reference's origin (-0.5, -0.5, 0), z
up (the reference's gravity is (0, 0, -9.81), `solver.py:126`), 8 particles per source cell seeded
by the reference's own generator (`numpy.random.default_rng(0)`, `solver.py:146-158`).

Scenes named after a benchmark configuration are that configuration as the reference can express
it: the liquid extents and collider of the configuration with its y-up axes turned to z-up, the
reference's whole-cell jitter instead of 2x2x2 sub-cell jitter, and the reference's fixed W-cycle
count (`settings.iterations`) instead of a residual tolerance.
"""

from __future__ import annotations

import hashlib
import json

import numpy as np

from continuum_liquid_b200.scenes import icosphere

IDENTITY = np.eye(4).tolist()


def box_triangles(lo, hi) -> np.ndarray:
    """Twelve triangles of an axis-aligned box (world space)."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], dtype=np.float32)
    faces = [(0, 1, 2), (0, 2, 3), (4, 6, 5), (4, 7, 6), (0, 4, 5), (0, 5, 1),
             (3, 2, 6), (3, 6, 7), (0, 3, 7), (0, 7, 4), (1, 5, 6), (1, 6, 2)]
    return v[np.array(faces)]


def entry(name: str, triangles: np.ndarray) -> dict:
    return {"object_name": name, "mesh_file": f"{name}.usdc", "matrix_world": IDENTITY,
            "triangles": np.ascontiguousarray(triangles, dtype=np.float32)}


def config(n: int, frames: int, sources: list, obstacles: list, fps: int = 240, substeps: int = 0,
           iterations: int = 1) -> dict:
    return {
        "meta": {},
        "simulation": {
            "output_path": "bake",
            "domain": {"resolution": 1.0 / n, "size": {"x": 1.0, "y": 1.0, "z": 1.0}},
            "physics": {"water": {"density": 1000.0, "viscosity": 1e-6},
                        "air": {"density": 1.0, "viscosity": 1.5e-5}},
            "settings": {"solver_backend": "GPU", "compute_devices": [{"platform_index": 0, "device_index": 0}],
                         "start_frame": 0, "end_frame": frames, "fps": fps, "substeps": substeps,
                         "iterations": iterations},
            "sources": sources,
            "obstacles": [{"geometry_inputs": [o]} for o in obstacles],
        },
    }


def _block(lo, hi):
    return [{"type": "GEOMETRY", "particle_density": 8, "geometry_inputs": [entry("block", box_triangles(lo, hi))]}]


def _pool_and_ball(ball_subdivisions: int, depth: float = 0.3):
    return [
        {"type": "GEOMETRY", "particle_density": 8,
         "geometry_inputs": [entry("pool", box_triangles((-0.5, -0.5, 0.0), (0.5, 0.5, depth)))]},
        {"type": "GEOMETRY", "particle_density": 8, "velocity": (0.0, 0.0, -2.0),
         "geometry_inputs": [entry("ball", icosphere(ball_subdivisions, 0.15, (0.0, 0.0, 0.7)))]},
    ]


def scene(name: str) -> dict:
    """The config of one named scene."""
    if name == "dam_break_16":
        return config(16, 5, _block((-0.5, -0.5, 0.0), (-0.1, -0.1, 0.6)), [])
    if name == "collider_pool_20":
        return config(20, 6, _pool_and_ball(2, depth=0.2), [entry("collider", icosphere(2, 0.15, (-0.2, 0.1, 0.15)))],
                      iterations=2)
    if name == "sources_24":
        sources = [
            {"type": "GEOMETRY", "particle_density": 8,
             "geometry_inputs": [entry("liquid", box_triangles((-0.45, -0.45, 0.05), (0.0, 0.0, 0.4)))]},
            {"type": "INFLOW", "particle_density": 8, "velocity": (0.0, 0.0, -1.0),
             "geometry_inputs": [entry("inflow", box_triangles((0.1, 0.1, 0.7), (0.3, 0.3, 0.85)))]},
            {"type": "OUTFLOW", "geometry_inputs": [entry("outflow", box_triangles((0.3, -0.45, 0.04),
                                                                                    (0.45, -0.3, 0.2)))]},
        ]
        obstacles = [entry("wall", box_triangles((-0.1, 0.2, 0.04), (0.05, 0.35, 0.3)))]
        return config(24, 4, sources, obstacles, fps=24, substeps=1)
    if name == "config1_dam_break_64":
        # 64^3 dam break: liquid [0,0.4] x [0,0.4] x [0,0.6] of the domain (height along z), 120 steps
        return config(64, 120, _block((-0.5, -0.5, 0.0), (-0.1, -0.1, 0.6)), [])
    if name == "config2_collider_pool_128":
        # 128^3: pool of depth 0.3, a ball of radius 0.15 at height 0.7 falling at 2 m/s, the
        # icosphere collider (subdivision 4, 5120 triangles, radius 0.12) at (0.3, 0.6, 0.15)
        return config(128, 2, _pool_and_ball(3), [entry("collider", icosphere(4, 0.12, (-0.2, 0.1, 0.15)))])
    if name == "config3_block_256":
        # 256^3: liquid [0,0.5] x [0,0.5] x [0,0.7] of the domain, the first step
        return config(256, 1, _block((-0.5, -0.5, 0.0), (0.0, 0.0, 0.7)), [])
    raise KeyError(name)


SMALL = ("dam_break_16", "collider_pool_20", "sources_24")
LARGE = ("config1_dam_break_64", "config2_collider_pool_128", "config3_block_256")


def meshes(cfg: dict) -> dict[str, np.ndarray]:
    """mesh_file name -> triangles, for the reference run."""
    sim = cfg["simulation"]
    entries = [e for s in sim.get("sources") or () for e in s.get("geometry_inputs") or ()]
    entries += [e for o in sim.get("obstacles") or () for e in o.get("geometry_inputs") or ()]
    return {e["mesh_file"]: e["triangles"] for e in entries}


def config_digest(cfg: dict) -> str:
    """A digest of a config (numbers and triangles), stored in each fixture to detect drift."""
    h = hashlib.sha256()

    def walk(value):
        if isinstance(value, dict):
            for key in sorted(value):
                h.update(key.encode())
                walk(value[key])
        elif isinstance(value, (list, tuple)):
            for item in value:
                walk(item)
        elif isinstance(value, np.ndarray):
            h.update(np.ascontiguousarray(value).tobytes())
        else:
            h.update(json.dumps(value).encode())

    walk(cfg)
    return h.hexdigest()[:24]


def digest(array: np.ndarray) -> str:
    """sha256 of an array's values (dtype, shape and bytes; floats with -0 folded into +0)."""
    a = np.ascontiguousarray(array)
    if a.dtype.kind == "f":
        a = a + a.dtype.type(0)
    h = hashlib.sha256(f"{a.dtype.str}{a.shape}".encode())
    h.update(a.tobytes())
    return h.hexdigest()[:32]
