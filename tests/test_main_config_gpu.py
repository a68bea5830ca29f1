"""The add-on's entry point end to end (Solver/General/main.py main(config)): a small bake with a
liquid block, an inflow, an outflow and a solid box, run by this backend to completion; the particle
cache and the stats messages come out in the reference's formats and the sources act every step."""

from __future__ import annotations

import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def box_triangles(lo, hi):
    """Twelve triangles of an axis-aligned box (world space)."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], dtype=np.float32)
    faces = [(0, 1, 2), (0, 2, 3), (4, 6, 5), (4, 7, 6), (0, 4, 5), (0, 5, 1),
             (3, 2, 6), (3, 6, 7), (0, 3, 7), (0, 7, 4), (1, 5, 6), (1, 6, 2)]
    return v[np.array(faces)]


def test_bake_with_dynamic_sources(tmp_path):
    from continuum_liquid_b200.general import main as general

    # the domain is [-0.5, 0.5] x [-0.5, 0.5] x [0, 1] in world space (origin (-x/2, -y/2, 0))
    entry = lambda lo, hi: {"object_name": "box", "triangles": box_triangles(lo, hi)}  # noqa: E731
    config = {
        "meta": {},
        "simulation": {
            "output_path": str(tmp_path / "bake"),
            "domain": {"resolution": 1.0 / 24.0, "size": {"x": 1.0, "y": 1.0, "z": 1.0}},
            "physics": {"water": {"density": 1000.0, "viscosity": 1e-6}},
            "settings": {"start_frame": 1, "end_frame": 5, "fps": 24, "substeps": 1, "flip_ratio": 0.95,
                         "tolerance": 1e-6, "gravity": (0.0, 0.0, -9.81)},
            "sources": [
                {"type": "GEOMETRY", "particle_density": 8, "geometry_inputs": [entry((-0.45, -0.45, 0.05), (0.0, 0.0, 0.4))]},
                {"type": "INFLOW", "particle_density": 8, "velocity": (0.0, 0.0, -1.0),
                 "geometry_inputs": [entry((0.1, 0.1, 0.7), (0.3, 0.3, 0.85))]},
                {"type": "OUTFLOW", "geometry_inputs": [entry((0.3, -0.45, 0.04), (0.45, -0.3, 0.2))]},
            ],
            "obstacles": [{"geometry_inputs": [entry((-0.1, 0.2, 0.04), (0.05, 0.35, 0.3))]}],
        },
    }
    messages = []
    general.set_message_callback(messages.append)
    try:
        general.main(config)
    finally:
        general.clear_message_callback()
    stats = [m for m in messages if m.get("type") == "stats"]
    assert [m["frame"] for m in stats] == [0, 1, 2, 3, 4]
    counts = [m["particle_count"] for m in stats]
    assert counts[-1] > counts[0]  # the inflow keeps adding particles
    assert all(m["solve"]["rel_residual"] <= 1e-6 for m in stats[1:])
    cache = json.loads((tmp_path / "bake" / "particle_cache.json").read_text())
    frames = sorted((tmp_path / "bake" / "particles").glob("particles_*.bin"))
    assert len(frames) == 5 and cache["version"] == 2
    last = np.fromfile(frames[-1], dtype=np.float32).reshape(-1, 3)
    assert len(last) == counts[-1] and np.isfinite(last).all()
