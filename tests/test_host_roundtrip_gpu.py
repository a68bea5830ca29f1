"""FlipSolver.step_host: the per-step host round trip of the particle state (solver.py:252-306) with
the copies split into pieces on two streams gives exactly the state of plain device steps."""
import numpy as np
import pytest
import torch

from continuum_liquid_b200 import scenes, solver


def _solver(backend, s):
    opts = solver.StepOptions(flip_ratio=0.95, tol=1e-6, gravity=s.gravity)
    pos, vel = scenes.seed_particles(s)
    return solver.FlipSolver(backend, s.grid_shape, s.dx, pos, vel, dt=s.dt, options=opts)


@pytest.mark.gpu
@pytest.mark.parametrize("chunks", [1, 3, 8])
def test_step_host_equals_device_steps(backend, chunks):
    s = scenes.block(32)
    a, b = _solver(backend, s), _solver(backend, s)
    host_pos = torch.empty((b.n, 3), dtype=torch.float32, pin_memory=True)
    host_vel = torch.empty((b.n, 3), dtype=torch.float32, pin_memory=True)
    host_pos.copy_(b.particles[: b.n])
    host_vel.copy_(b.particle_velocity[: b.n])
    torch.cuda.synchronize()
    for _ in range(4):
        a.step()
        b.step_host(host_pos, host_vel, chunks=chunks)
    torch.cuda.synchronize()
    assert np.array_equal(host_pos.numpy(), a.positions())
    assert np.array_equal(host_vel.numpy(), a.velocities())
    assert np.array_equal(b.positions(), a.positions())
    # a plain step after the round trips continues from the downloaded state
    a.step()
    b.step()
    assert np.array_equal(b.positions(), a.positions())
    assert backend.device_error() == 0


@pytest.mark.gpu
def test_step_host_rejects_pageable_or_misshapen_buffers(backend):
    s = scenes.block(24)
    b = _solver(backend, s)
    with pytest.raises(ValueError):
        b.step_host(torch.zeros((b.n, 3)), torch.zeros((b.n, 3)))
    pinned = torch.zeros((b.n + 1, 3), dtype=torch.float32, pin_memory=True)
    with pytest.raises(ValueError):
        b.step_host(pinned, pinned)
