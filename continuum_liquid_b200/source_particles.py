"""Host-side particle sources (mirrors Solver/Kernel/source_particles.py).

Sources are voxelised on the device and their masks downloaded once; seeding, inflow top-up and
outflow removal then run on the host with numpy, exactly where the reference runs them.
"""

from __future__ import annotations

import numpy as np

FIELD_DTYPE = np.float32


def download_static_masks(queue, sources, obstacle_mask_device, grid_shape):
    """source_particles.py:7-18: host boolean copies of the static masks."""
    obstacle = obstacle_mask_device.cpu().numpy().astype(np.bool_)
    result = []
    for source in sources:
        entry = {key: value for key, value in source.items() if key != "mask_device"}
        entry["mask"] = source["mask_device"].cpu().numpy().astype(np.bool_)
        result.append(entry)
    return result, obstacle


def particle_cells(positions, delta, grid_shape):
    """source_particles.py:21-25: clamp(floor(p / delta), 0, n - 1)."""
    if len(positions) == 0:
        return np.empty((0, 3), dtype=np.int32)
    cells = np.floor(np.asarray(positions) / delta).astype(np.int32)
    return np.clip(cells, 0, np.asarray(grid_shape, dtype=np.int32) - 1)


def mask_membership(positions, mask, delta):
    """source_particles.py:28-34."""
    cells = particle_cells(positions, delta, mask.shape)
    if len(cells) == 0:
        return np.zeros(0, dtype=np.bool_)
    return mask[cells[:, 0], cells[:, 1], cells[:, 2]]


def remove_masked(particles, velocities, mask, delta):
    """source_particles.py:37-39: drop particles inside an outflow mask."""
    keep = ~mask_membership(particles, mask, delta)
    return particles[keep], velocities[keep]


def fill_source(particles, velocities, source, obstacle_mask, delta, rng):
    """source_particles.py:42-75: top every non-solid source cell up to ``particle_density``
    particles, each new one uniform in its cell, with the source velocity."""
    target = max(1, int(source.get("particle_density", 8)))
    source_mask = np.asarray(source["mask"], dtype=np.bool_) & ~obstacle_mask
    cells = np.argwhere(source_mask)
    if len(cells) == 0:
        return particles, velocities
    counts = np.zeros(source_mask.shape, dtype=np.int64)
    occupied = particle_cells(particles, delta, source_mask.shape)
    if len(occupied):
        flat = np.ravel_multi_index(occupied.T, source_mask.shape)
        counts.flat[:] = np.bincount(flat, minlength=source_mask.size)
    missing = np.maximum(0, target - counts[tuple(cells.T)])
    spawn = np.repeat(cells, missing, axis=0)
    if len(spawn) == 0:
        return particles, velocities
    new_positions = (spawn + rng.random((len(spawn), 3))) * delta
    velocity = np.asarray(source.get("velocity", (0.0, 0.0, 0.0)), dtype=FIELD_DTYPE)
    new_velocities = np.broadcast_to(velocity, new_positions.shape)
    return (
        np.ascontiguousarray(np.concatenate((particles, new_positions)), dtype=FIELD_DTYPE),
        np.ascontiguousarray(np.concatenate((velocities, new_velocities)), dtype=FIELD_DTYPE),
    )


def apply_sources(particles, velocities, sources, obstacle_mask, delta, rng, initial=False):
    """source_particles.py:78-92: outflows first, then inflows (and geometry sources initially)."""
    for source in sources:
        if source.get("type") == "OUTFLOW":
            particles, velocities = remove_masked(particles, velocities, source["mask"], delta)
    for source in sources:
        kind = source.get("type")
        if kind == "INFLOW" or (initial and kind == "GEOMETRY"):
            particles, velocities = fill_source(particles, velocities, source, obstacle_mask, delta, rng)
    return particles, velocities


__all__ = ["download_static_masks", "particle_cells", "mask_membership", "remove_masked", "fill_source",
           "apply_sources"]
