"""Particle binning, counting sort, P2G and G2P stages (mirrors Solver/Kernel/particles.py).

Function names and argument order follow the reference; ``kernels`` is a ``Backend``, ``queue`` a
``torch.cuda.Stream`` (or None for the current stream) and every ``cl.Buffer`` a contiguous CUDA
tensor of the same dtype and shape.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .backend import Backend
from .colliders import motion_arg

FIELD_DTYPE = np.float32


@dataclass
class SortScratch:
    """Workspace of the stable counting sort: the scan's look-back state and four int32[N] arrays
    (bin key and rank per particle, slot permutation and slot keys). Takes the place of the
    reference's block-sum pyramid (particles.py:10-36)."""

    scan: torch.Tensor
    keys: torch.Tensor
    ranks: torch.Tensor
    perm: torch.Tensor
    slot_keys: torch.Tensor


def _device_of(context) -> torch.device:
    if isinstance(context, Backend):
        return context.device
    if isinstance(context, torch.device):
        return context
    return torch.device("cuda", 0)


def create_particle_sort_buffers(context, grid_shape, particle_count_total):
    """particles.py:10-36: double buffers and scratch for cell sorting.

    Returns ``(particle_work, particle_velocity_work, bin_counts, scan_outputs, scan_sums)`` like the
    reference; ``scan_outputs`` is ``[bin_offsets]`` and ``scan_sums`` is a one-element list holding
    the ``SortScratch``.
    """
    device = _device_of(context)
    cell_count = int(np.prod(grid_shape))
    n = max(1, int(particle_count_total))
    scan_bytes = Backend.scan_scratch_bytes_static(cell_count)
    particle_work = torch.empty((n, 3), dtype=torch.float32, device=device)
    particle_velocity_work = torch.empty((n, 3), dtype=torch.float32, device=device)
    bin_counts = torch.zeros(cell_count, dtype=torch.int32, device=device)
    offsets = torch.zeros(cell_count, dtype=torch.int32, device=device)
    scratch = SortScratch(
        scan=torch.zeros(scan_bytes, dtype=torch.uint8, device=device),
        keys=torch.empty(n, dtype=torch.int32, device=device),
        ranks=torch.empty(n, dtype=torch.int32, device=device),
        perm=torch.empty(n, dtype=torch.int32, device=device),
        slot_keys=torch.empty(n, dtype=torch.int32, device=device),
    )
    return particle_work, particle_velocity_work, bin_counts, [offsets], [scratch]


def count_particles_per_cell(kernels: Backend, queue, particles, bin_counts, particle_count_total, grid_shape, dx,
                             keys=None, ranks=None):
    """particles.cl:44-59 (accumulates into bin_counts; zero-fill first as particles.py:146 does)."""
    nx, ny, nz = grid_shape
    kernels.call("clb_count_particles_per_cell", particles, bin_counts, keys, ranks, int(particle_count_total),
                 float(FIELD_DTYPE(1.0 / float(dx))), nx, ny, nz, stream=queue)
    return bin_counts


def exclusive_prefix_sum(kernels: Backend, queue, values, outputs, sums, count, total=None):
    """particles.py:39-70: exclusive scan of ``values`` into ``outputs[0]`` (single pass)."""
    scratch = sums[0].scan if isinstance(sums[0], SortScratch) else sums[0]
    kernels.call("clb_exclusive_prefix_sum", values, outputs[0], total, int(count), scratch, int(scratch.numel()),
                 stream=queue)
    return outputs[0]


def sort_particles(kernels: Backend, queue, particles, particle_velocity, particles_sorted, particle_velocity_sorted,
                   bin_offsets, bin_counts, scratch: SortScratch, particle_count_total):
    """particles.cl:110-133 as a stable counting-sort scatter (order within a bin = input order)."""
    kernels.call("clb_sort_particles", particles, particle_velocity, particles_sorted, particle_velocity_sorted,
                 bin_offsets, bin_counts, scratch.keys, scratch.ranks, scratch.perm, scratch.slot_keys,
                 int(particle_count_total), stream=queue)


def particle_to_grid_gather(kernels: Backend, queue, particles, particle_velocity, bin_offsets, bin_counts, velocity,
                            fluid_fraction, grid_shape, dx, particles_per_cell, tiled: bool = False):
    """particles.cl:135-227 (dispatched as particles.py:194-215). ``tiled``: the tiled scatter that
    visits each particle once (every weight the reference's, each cell's sums in another fixed order:
    equal to float rounding, not bit for bit)."""
    nx, ny, nz = grid_shape
    u, v, w = velocity
    name = "clb_particle_to_grid_gather_tiled" if tiled else "clb_particle_to_grid_gather"
    kernels.call(name, particles, particle_velocity, bin_offsets, bin_counts, u, v, w,
                 fluid_fraction, float(FIELD_DTYPE(1.0 / float(dx))), float(FIELD_DTYPE(1.0 / particles_per_cell)), nx, ny,
                 nz, stream=queue)


def particle_to_grid(
    kernels: Backend,
    queue,
    particles,
    particle_velocity,
    particle_work,
    particle_velocity_work,
    velocity,
    particle_bin_counts,
    particle_bin_scan_outputs,
    particle_bin_scan_sums,
    fluid_fraction,
    particle_count_total,
    grid_shape,
    dx,
    particles_per_cell,
    tiled: bool = False,
):
    """particles.py:73-171: count, scan, sort into the work buffers, swap, gather.

    Returns ``(particles, particle_velocity, particle_work, particle_velocity_work, velocity,
    fluid_fraction)`` with the particle buffers swapped, exactly like the reference. ``tiled`` selects
    the tiled gather (see ``particle_to_grid_gather``); binning and sort are the same either way.
    """
    nx, ny, nz = grid_shape
    u, v, w = velocity
    scratch: SortScratch = particle_bin_scan_sums[0]
    kernels.call(
        "clb_particle_to_grid_tiled" if tiled else "clb_particle_to_grid",
        particles,
        particle_velocity,
        particle_work,
        particle_velocity_work,
        u,
        v,
        w,
        fluid_fraction,
        particle_bin_counts,
        particle_bin_scan_outputs[0],
        scratch.keys,
        scratch.ranks,
        scratch.perm,
        scratch.slot_keys,
        scratch.scan,
        int(scratch.scan.numel()),
        int(particle_count_total),
        float(FIELD_DTYPE(1.0 / float(dx))),
        float(FIELD_DTYPE(1.0 / particles_per_cell)),
        nx,
        ny,
        nz,
        stream=queue,
    )
    particles, particle_work = particle_work, particles
    particle_velocity, particle_velocity_work = particle_velocity_work, particle_velocity
    return particles, particle_velocity, particle_work, particle_velocity_work, velocity, fluid_fraction


def grid_to_particle(kernels: Backend, queue, particle_velocity, particles, velocity, old_velocity,
                     particle_count_total, grid_shape, dx, flip_ratio: float = 1.0):
    """particles.py:174-206 (+ FLIP/PIC blend; ``flip_ratio=1`` is the reference's pure FLIP)."""
    nx, ny, nz = grid_shape
    u, v, w = velocity
    ou, ov, ow = old_velocity
    kernels.call("clb_grid_to_particle", particle_velocity, particles, u, v, w, ou, ov, ow, int(particle_count_total),
                 float(FIELD_DTYPE(1.0 / float(dx))), nx, ny, nz, float(FIELD_DTYPE(flip_ratio)), stream=queue)
    return particle_velocity


def advect_particles(kernels: Backend, queue, particles, particle_velocity, particle_count_total, dt):
    """particles.py:209-225."""
    kernels.call("clb_advect_particles", particles, particle_velocity, int(particle_count_total),
                 float(FIELD_DTYPE(dt)), stream=queue)
    return particles


def particle_update(kernels: Backend, queue, particles, particle_velocity, velocity, old_velocity, obstacle,
                    particle_count_total, grid_shape, dx, dt, flip_ratio: float = 1.0, previous_particles=None,
                    motion=None, bins=None):
    """solver.py:453-510 fused: G2P, previous-position copy, advection, domain and obstacle BCs.

    ``obstacle`` may be None when the scene has no collider (the obstacle BC is then a no-op in the
    reference as well). ``previous_particles`` receives the pre-advection positions when given.
    ``motion`` (with an obstacle): the collider moves rigidly (``colliders.RigidMotion.parameters``).
    ``bins``: ``(bin_offsets, bin_counts)`` of the particles' counting sort when they are still sorted
    by bin; the update then walks the bins tile by tile (``clb_particle_update_tiled``, same values).
    """
    nx, ny, nz = grid_shape
    u, v, w = velocity
    ou, ov, ow = old_velocity
    if bins is not None:
        offsets, counts = bins
        kernels.call("clb_particle_update_tiled", particles, particle_velocity, previous_particles, u, v, w, ou, ov, ow,
                     obstacle, offsets, counts, int(particle_count_total), float(FIELD_DTYPE(1.0 / float(dx))), nx, ny,
                     nz, float(FIELD_DTYPE(flip_ratio)), float(FIELD_DTYPE(dt)),
                     float(FIELD_DTYPE(1.001 * float(dx))), float(FIELD_DTYPE((nx - 1.001) * float(dx))),
                     float(FIELD_DTYPE((ny - 1.001) * float(dx))), float(FIELD_DTYPE((nz - 1.001) * float(dx))),
                     None if motion is None else motion_arg(motion), stream=queue)
        return particles, particle_velocity
    extra = () if motion is None else (motion_arg(motion),)
    kernels.call(
        "clb_particle_update" if motion is None else "clb_particle_update_moving",
        particles,
        particle_velocity,
        previous_particles,
        u,
        v,
        w,
        ou,
        ov,
        ow,
        obstacle,
        int(particle_count_total),
        float(FIELD_DTYPE(1.0 / float(dx))),
        nx,
        ny,
        nz,
        float(FIELD_DTYPE(flip_ratio)),
        float(FIELD_DTYPE(dt)),
        float(FIELD_DTYPE(1.001 * float(dx))),
        float(FIELD_DTYPE((grid_shape[0] - 1.001) * float(dx))),
        float(FIELD_DTYPE((grid_shape[1] - 1.001) * float(dx))),
        float(FIELD_DTYPE((grid_shape[2] - 1.001) * float(dx))),
        *extra,
        stream=queue,
    )
    return particles, particle_velocity
