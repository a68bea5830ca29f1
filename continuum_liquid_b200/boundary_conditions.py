"""Boundary-condition stages (mirrors Solver/Kernel/boundary_conditions.py)."""

from __future__ import annotations

import numpy as np

from .backend import Backend
from .colliders import motion_arg

FIELD_DTYPE = np.float32


def neumann_domain_bc(kernels: Backend, queue, pressure, grid_shape):
    """boundary_conditions.py:22-33 (boundary_conditions.cl:18-31)."""
    nx, ny, nz = grid_shape
    kernels.call("clb_neumann_domain_bc", pressure, nx, ny, nz, stream=queue)
    return pressure


def grid_domain_bc(kernels: Backend, queue, velocity, grid_shape):
    """boundary_conditions.py:36-50 (boundary_conditions.cl:33-67)."""
    nx, ny, nz = grid_shape
    u, v, w = velocity
    kernels.call("clb_grid_domain_bc", u, v, w, nx, ny, nz, stream=queue)
    return velocity


def grid_obstacle_bc(kernels: Backend, queue, velocity, fluid_fraction, obstacle, grid_shape, motion=None, dx=None):
    """boundary_conditions.py:53-79: obstacle faces and fluid fraction, then the tangential
    extrapolation into solid cells as a second launch. ``motion`` (the 9 parameters of
    ``colliders.RigidMotion.parameters``, with the cell size ``dx``): a moving collider, whose solid
    faces take its velocity (no counterpart in the reference)."""
    nx, ny, nz = grid_shape
    u, v, w = velocity
    if motion is None:
        kernels.call("clb_grid_obstacle_bc", u, v, w, fluid_fraction, obstacle, nx, ny, nz, stream=queue)
    else:
        kernels.call("clb_grid_obstacle_bc_moving", u, v, w, fluid_fraction, obstacle, nx, ny, nz, motion_arg(motion),
                     float(FIELD_DTYPE(dx)), stream=queue)
    return velocity, fluid_fraction


def particle_domain_bc(kernels: Backend, queue, particles, particle_velocity, particle_count_total, grid_shape, dx):
    """boundary_conditions.py:82-103 (walls at 1.001 dx and (n - 1.001) dx)."""
    kernels.call(
        "clb_particle_domain_bc",
        particles,
        particle_velocity,
        int(particle_count_total),
        float(FIELD_DTYPE(1.001 * float(dx))),
        float(FIELD_DTYPE((grid_shape[0] - 1.001) * float(dx))),
        float(FIELD_DTYPE((grid_shape[1] - 1.001) * float(dx))),
        float(FIELD_DTYPE((grid_shape[2] - 1.001) * float(dx))),
        stream=queue,
    )
    return particles, particle_velocity


def particle_obstacle_bc(kernels: Backend, queue, particles, previous_particles, particle_velocity, obstacle,
                         particle_count_total, grid_shape, dx, motion=None):
    """boundary_conditions.py:106-132 (boundary_conditions.cl:175-264). ``motion``: a moving
    collider; only the velocity relative to it loses its inward component."""
    nx, ny, nz = grid_shape
    if motion is None:
        kernels.call("clb_particle_obstacle_bc", particles, previous_particles, particle_velocity, obstacle,
                     int(particle_count_total), float(FIELD_DTYPE(1.0 / float(dx))), nx, ny, nz, stream=queue)
    else:
        kernels.call("clb_particle_obstacle_bc_moving", particles, previous_particles, particle_velocity, obstacle,
                     int(particle_count_total), float(FIELD_DTYPE(1.0 / float(dx))), nx, ny, nz, motion_arg(motion),
                     stream=queue)
    return particles, particle_velocity
