"""ORACLE -- test infrastructure only; never imported by the product package.

Host-side particle sources of the reference, restated with numpy in the reference's order of
operations (`Solver/Kernel/source_particles.py`), so that a bake restated here draws from
`numpy.random.default_rng` exactly as the reference does: the same cells in the same order, the
same number of draws, the same float64 arithmetic rounded to float32. The product seeds and tops
up particles on the device (`continuum_liquid_b200.source_particles.DeviceSources`); tests compare
it with this restatement and with the reference's own bakes (tests/golden/ref_*.npz).
"""

from __future__ import annotations

import numpy as np

FIELD_DTYPE = np.float32


def particle_cells(positions, delta, grid_shape):
    """source_particles.py:21-25: the cell of each particle, floor(p / delta) clamped to the grid."""
    if len(positions) == 0:
        return np.empty((0, 3), dtype=np.int32)
    cells = np.floor(np.asarray(positions) / delta).astype(np.int32)
    return np.clip(cells, 0, np.asarray(grid_shape, dtype=np.int32) - 1)


def mask_membership(positions, mask, delta):
    """source_particles.py:28-34: whether each particle's cell is set in ``mask``."""
    cells = particle_cells(positions, delta, mask.shape)
    if len(cells) == 0:
        return np.zeros(0, dtype=np.bool_)
    return mask[cells[:, 0], cells[:, 1], cells[:, 2]]


def remove_masked(particles, velocities, mask, delta):
    """source_particles.py:37-39: the particles outside ``mask``, in their order."""
    keep = ~mask_membership(particles, mask, delta)
    return particles[keep], velocities[keep]


def fill_source(particles, velocities, source, obstacle_mask, delta, rng):
    """source_particles.py:42-75: every source cell that is not solid gets new particles up to the
    source's density; cells in argwhere (flat) order, each new particle (cell + U[0,1)^3) * delta
    in float64 from three consecutive draws, then rounded to float32; the source velocity."""
    density = max(1, int(source.get("particle_density", 8)))
    region = np.asarray(source["mask"], dtype=np.bool_) & ~obstacle_mask
    cells = np.argwhere(region)
    if len(cells) == 0:
        return particles, velocities
    present = np.zeros(region.shape, dtype=np.int32)
    occupied = particle_cells(particles, delta, region.shape)
    if len(occupied):
        flat = np.ravel_multi_index(occupied.T, region.shape)
        present.flat[:] = np.bincount(flat, minlength=region.size).astype(np.int32, copy=False)
    missing = np.maximum(0, density - present[tuple(cells.T)])
    spawn = np.repeat(cells, missing, axis=0)
    if len(spawn) == 0:
        return particles, velocities
    new_positions = (spawn + rng.random((len(spawn), 3))) * delta
    velocity = np.asarray(source.get("velocity", (0.0, 0.0, 0.0)), dtype=FIELD_DTYPE)
    new_velocities = np.broadcast_to(velocity, new_positions.shape).copy()
    return (np.ascontiguousarray(np.concatenate((particles, new_positions)), dtype=FIELD_DTYPE),
            np.ascontiguousarray(np.concatenate((velocities, new_velocities)), dtype=FIELD_DTYPE))


def apply_sources(particles, velocities, sources, obstacle_mask, delta, rng, initial=False):
    """source_particles.py:78-92: every outflow first, then each inflow in order (and, on the
    initial fill, each geometry source)."""
    for source in sources:
        if source.get("type") == "OUTFLOW":
            particles, velocities = remove_masked(particles, velocities, source["mask"], delta)
    for source in sources:
        kind = source.get("type")
        if kind == "INFLOW" or (initial and kind == "GEOMETRY"):
            particles, velocities = fill_source(particles, velocities, source, obstacle_mask, delta, rng)
    return particles, velocities
