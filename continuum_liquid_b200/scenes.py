"""Seeded synthetic scenes for the benchmark configurations.

The reference has no public dataset or benchmark scenes; these generated inputs stand in for them.
Grids include the ghost layer, as ``nx = int(Lx / resolution)`` does in the reference
(solver.py:109-117). Particles live in grid-local coordinates [0, n*dx]; a cell (i, j, k) covers
[i*dx, (i+1)*dx) and is seeded only when it is an interior cell whose centre lies in the liquid
region and which is not solid (source_particles.py:42-75 seeds interior, non-obstacle cells).
Each seeded cell receives 8 particles, one uniformly jittered inside each of its 2x2x2 sub-cells,
from ``numpy.random.default_rng(seed)``. Collider meshes are icospheres in world coordinates with
the reference's domain origin (-Lx/2, -Ly/2, 0) (voxelise_mesh.py:140).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable

import numpy as np

Region = Callable[[np.ndarray, np.ndarray, np.ndarray], np.ndarray]


def icosphere(subdivisions: int, radius: float = 1.0, centre=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Triangles (20 * 4**subdivisions, 3, 3) float32 of a subdivided icosahedron."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    v = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache: dict[tuple[int, int], int] = {}

        def midpoint(a: int, b: int) -> int:
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[key] = len(v) - 1
            return cache[key]

        new_faces = []
        for a, b, c in faces:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            new_faces += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = new_faces
    verts_arr = np.asarray(v) * float(radius) + np.asarray(centre, dtype=np.float64)
    return np.ascontiguousarray(verts_arr[np.asarray(faces)], dtype=np.float32)


def box(lo, hi) -> Region:
    lo, hi = np.asarray(lo, dtype=np.float64), np.asarray(hi, dtype=np.float64)
    return lambda x, y, z: (x >= lo[0]) & (x <= hi[0]) & (y >= lo[1]) & (y <= hi[1]) & (z >= lo[2]) & (z <= hi[2])


def ball(centre, radius) -> Region:
    c = np.asarray(centre, dtype=np.float64)
    return lambda x, y, z: (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 <= radius * radius


@dataclass
class Source:
    region: Region
    velocity: tuple[float, float, float] = (0.0, 0.0, 0.0)


@dataclass
class Scene:
    """A simulation setup: grid, liquid sources, colliders and time stepping."""

    name: str
    grid_shape: tuple[int, int, int]
    dx: float
    sources: list[Source]
    obstacles: list[np.ndarray] = field(default_factory=list)  # world-space triangles per mesh
    gravity: tuple[float, float, float] = (0.0, -9.81, 0.0)
    dt: float = 1.0 / 240.0
    flip_ratio: float = 0.95
    rho: float = 1000.0
    nu: float = 1.0e-6
    steps: int = 100
    min_size: int = 8
    seed: int = 0
    particles_per_cell: int = 8

    @property
    def origin(self) -> tuple[float, float, float]:
        return (-0.5 * self.grid_shape[0] * self.dx, -0.5 * self.grid_shape[1] * self.dx, 0.0)

    @property
    def cells(self) -> int:
        return int(np.prod(self.grid_shape))


def seed_particles(scene: Scene, obstacle_mask: np.ndarray | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Positions and velocities (float32, (N,3)) for the scene's sources, skipping solid cells."""
    nx, ny, nz = scene.grid_shape
    dx = scene.dx
    centres = [(np.arange(n, dtype=np.float64) + 0.5) * dx for n in (nx, ny, nz)]
    X, Y, Z = np.meshgrid(*centres, indexing="ij")
    interior = np.zeros(scene.grid_shape, dtype=bool)
    interior[1:-1, 1:-1, 1:-1] = True
    taken = np.zeros(scene.grid_shape, dtype=bool)
    rng = np.random.default_rng(scene.seed)
    sub = np.array([[a, b, c] for a in (0, 1) for b in (0, 1) for c in (0, 1)], dtype=np.float64)
    positions, velocities = [], []
    for source in scene.sources:
        sel = source.region(X, Y, Z) & interior & ~taken
        if obstacle_mask is not None:
            sel &= ~obstacle_mask.astype(bool)
        taken |= sel
        cells = np.argwhere(sel).astype(np.float64)
        if len(cells) == 0:
            continue
        jitter = rng.random((len(cells), 8, 3))
        pos = (cells[:, None, :] + (sub[None, :, :] + jitter) * 0.5) * dx
        positions.append(pos.reshape(-1, 3).astype(np.float32))
        velocities.append(np.broadcast_to(np.asarray(source.velocity, dtype=np.float32), (len(cells) * 8, 3)))
    if not positions:
        return np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32)
    return (np.ascontiguousarray(np.concatenate(positions)), np.ascontiguousarray(np.concatenate(velocities)))


def dam_break(n: int = 64, seed: int = 0) -> Scene:
    """Plain FLIP dam break: n^3 on the unit cube, block [0,0.4]x[0,0.6]x[0,0.4], 120 steps."""
    return Scene(f"dam_break_{n}", (n, n, n), 1.0 / n, [Source(box((0, 0, 0), (0.4, 0.6, 0.4)))], steps=120,
                 seed=seed)


def collider_pool(n: int = 128, seed: int = 0, subdivisions: int = 4) -> Scene:
    """Pool of depth 0.3 plus a falling sphere (r 0.15 at (0.5,0.7,0.5), v=(0,-2,0)) and a static
    icosphere collider (r 0.12 at (0.3,0.15,0.6)), 200 steps."""
    scene = Scene(f"collider_pool_{n}", (n, n, n), 1.0 / n,
                  [Source(box((0, 0, 0), (1, 0.3, 1))), Source(ball((0.5, 0.7, 0.5), 0.15), (0.0, -2.0, 0.0))],
                  steps=200, seed=seed)
    centre_local = np.array([0.3, 0.15, 0.6])
    scene.obstacles = [icosphere(subdivisions, 0.12, centre_local + np.asarray(scene.origin))]
    return scene


def block(n: int = 256, seed: int = 0) -> Scene:
    """Mixed-precision pressure case: n^3, block [0,0.5]x[0,0.7]x[0,0.5] (~23M particles at 256^3)."""
    return Scene(f"block_{n}", (n, n, n), 1.0 / n, [Source(box((0, 0, 0), (0.5, 0.7, 0.5)))], steps=100, seed=seed)


def uneven_batch(count: int = 32, seed: int = 0, sizes=(48, 64, 96, 128, 160)) -> list[Scene]:
    """Independent scenes of cubic sizes drawn from ``sizes``; each has a random axis-aligned liquid
    block filling 20-50% of the volume and one icosphere obstacle (subdivision 3, r in [0.08,0.2])."""
    rng = np.random.default_rng(seed)
    scenes = []
    for s in range(count):
        n = int(rng.choice(sizes))
        fraction = rng.uniform(0.2, 0.5)
        ext = np.clip(rng.uniform(0.4, 1.0, 3), 0.3, 1.0)
        ext = ext * (fraction / np.prod(ext)) ** (1.0 / 3.0)
        ext = np.clip(ext, 0.1, 1.0)
        lo = rng.uniform(0.0, 1.0 - ext)
        lo[1] = 0.0
        radius = float(rng.uniform(0.08, 0.2))
        centre = rng.uniform(radius + 0.05, 1.0 - radius - 0.05, 3)
        scene = Scene(f"uneven_{s}_{n}", (n, n, n), 1.0 / n, [Source(box(lo, lo + ext))], steps=200,
                      seed=seed * 1000 + s)
        scene.obstacles = [icosphere(3, radius, centre + np.asarray(scene.origin))]
        scenes.append(scene)
    return scenes
