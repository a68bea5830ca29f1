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


class DeviceSources:
    """Outflow removal and inflow top-up on the device, for the sources of a running simulation
    (apply_sources without ``initial``: outflows first, then each inflow in order). The results equal
    apply_sources on the host with the same random generator, which this class advances by the draws
    it uses; the particles never leave the GPU (only the counts are read back, to size the buffers).

    ``sources``: dicts with ``type`` ("INFLOW" / "OUTFLOW"), ``mask_device`` (uint8 grid tensor),
    ``particle_density`` and ``velocity`` as in the reference; ``obstacle``: uint8 grid tensor or None.
    """

    def __init__(self, kernels, sources, obstacle, grid_shape, delta, rng):
        import torch

        self.k = kernels
        self.grid_shape = tuple(int(x) for x in grid_shape)
        self.delta = float(delta)
        self.rng = rng
        dev = kernels.device
        cells = int(np.prod(self.grid_shape))
        self.cells = cells
        self.obstacle = obstacle
        outflows = [src["mask_device"] for src in sources if src.get("type") == "OUTFLOW"]
        self.outflow = None
        if outflows:
            combined = torch.zeros(self.grid_shape, dtype=torch.uint8, device=dev)
            for m in outflows:
                combined |= (m != 0).to(torch.uint8)
            self.outflow = combined
        self.inflows = [(src["mask_device"].to(torch.uint8).contiguous(), max(1, int(src.get("particle_density", 8))),
                         tuple(float(FIELD_DTYPE(c)) for c in src.get("velocity", (0.0, 0.0, 0.0))))
                        for src in sources if src.get("type") == "INFLOW"]
        self.counts = torch.zeros(cells, dtype=torch.int32, device=dev)
        self.missing = torch.zeros(cells, dtype=torch.int32, device=dev)
        self.offsets = torch.zeros(cells, dtype=torch.int32, device=dev)
        self.total = torch.zeros(1, dtype=torch.int32, device=dev)
        self.cell_scan = torch.zeros(kernels.scan_scratch_bytes(cells), dtype=torch.uint8, device=dev)
        self._keep = self._slots = self._particle_scan = None

    def _particle_buffers(self, n):
        import torch

        if self._keep is None or self._keep.numel() < n:
            size = max(1, n)
            dev = self.k.device
            self._keep = torch.zeros(size, dtype=torch.int32, device=dev)
            self._slots = torch.zeros(size, dtype=torch.int32, device=dev)
            self._particle_scan = torch.zeros(self.k.scan_scratch_bytes(size), dtype=torch.uint8, device=dev)

    def apply(self, sim) -> None:
        """Apply the sources to ``sim`` (a FlipSolver) in place."""
        k, nx_ny_nz = self.k, self.grid_shape
        delta32 = float(FIELD_DTYPE(self.delta))
        n = sim.n
        if self.outflow is not None and n > 0:
            self._particle_buffers(n)
            k.call("clb_source_keep", sim.particles, n, delta32, *nx_ny_nz, self.outflow, self._keep)
            k.call("clb_exclusive_prefix_sum", self._keep, self._slots, self.total, n, self._particle_scan,
                   int(self._particle_scan.numel()))
            k.call("clb_source_compact", sim.particles, sim.particle_velocity, self._keep, self._slots, n,
                   sim.particle_work, sim.particle_velocity_work)
            sim.particles, sim.particle_work = sim.particle_work, sim.particles
            sim.particle_velocity, sim.particle_velocity_work = sim.particle_velocity_work, sim.particle_velocity
            n = int(self.total.item())
        for mask, target, velocity in self.inflows:
            self.counts.zero_()
            k.call("clb_source_cell_counts", sim.particles, n, delta32, *nx_ny_nz, self.counts)
            k.call("clb_source_missing", self.counts, mask, self.obstacle, target, self.cells, self.missing)
            k.call("clb_exclusive_prefix_sum", self.missing, self.offsets, self.total, self.cells, self.cell_scan,
                   int(self.cell_scan.numel()))
            added = int(self.total.item())
            if added == 0:
                continue
            sim.ensure_capacity(n + added)
            st = self.rng.bit_generator.state["state"]
            state, inc = int(st["state"]), int(st["inc"])
            lo = (1 << 64) - 1
            k.call("clb_source_spawn", self.missing, self.offsets, *nx_ny_nz, self.delta, *velocity, state >> 64,
                   state & lo, inc >> 64, inc & lo, sim.particles[n:], sim.particle_velocity[n:])
            self.rng.bit_generator.advance(3 * added)
            n += added
        sim.n = n


__all__ = ["download_static_masks", "particle_cells", "mask_membership", "remove_masked", "fill_source",
           "apply_sources", "DeviceSources"]
