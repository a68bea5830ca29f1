"""Particle sources (the stage of Solver/Kernel/source_particles.py) on the device.

The reference voxelises its source meshes on the device, downloads the masks once and then seeds,
tops up and removes particles on the host with numpy, copying every particle to the host and back
before each step (solver.py:252-306). Here the initial fill, the inflows and the outflows run on the
GPU (``DeviceSources``) and draw the reference's random stream, so the particles are the ones the
reference's host code makes, bit for bit, without leaving the device.
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


class DeviceSources:
    """The reference's ``apply_sources`` (source_particles.py:78-92) on the device: every outflow
    first, then each inflow in order, and with ``initial`` each geometry source too (the initial
    fill, solver.py:146-158). A source cell that is not solid is topped up to the source's density;
    the new particles of a cell are placed in flat cell order, each at (cell + three consecutive
    draws of the generator) * delta in float64, rounded to float32, which is what the reference's
    numpy code computes. This class advances ``rng`` by the draws it uses, so host and device stay
    interchangeable; the particles never leave the GPU (only the counts are read back, to size the
    buffers).

    ``sources``: dicts with ``type`` ("GEOMETRY" / "INFLOW" / "OUTFLOW"), ``mask_device`` (uint8 grid
    tensor), ``particle_density`` and ``velocity`` as in the reference; ``obstacle``: uint8 grid
    tensor or None.
    """

    def __init__(self, kernels, sources, obstacle, grid_shape, delta, rng, initial: bool = False):
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
                        for src in sources
                        if src.get("type") == "INFLOW" or (initial and src.get("type") == "GEOMETRY")]
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
            sim.n = n  # the particles so far (outflows and earlier fills) survive a reallocation
            sim.ensure_capacity(n + added)
            st = self.rng.bit_generator.state["state"]
            state, inc = int(st["state"]), int(st["inc"])
            lo = (1 << 64) - 1
            k.call("clb_source_spawn", self.missing, self.offsets, *nx_ny_nz, self.delta, *velocity, state >> 64,
                   state & lo, inc >> 64, inc & lo, sim.particles[n:], sim.particle_velocity[n:])
            self.rng.bit_generator.advance(3 * added)
            n += added
        sim.n = n


__all__ = ["download_static_masks", "DeviceSources"]
