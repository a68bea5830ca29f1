"""Particle sources on the device (source_particles.DeviceSources) against the oracle's host
restatement of source_particles.py:37-92 (apply_sources) with the same random generator: bit-exact
particles, including buffer growth, the initial fill of geometry sources, and the same generator
state afterwards."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from continuum_liquid_b200 import solver, source_particles
from oracle import sources as host_sources_oracle

pytestmark = pytest.mark.gpu


def box_mask(shape, lo, hi):
    m = np.zeros(shape, dtype=np.uint8)
    m[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = 1
    return m


def test_device_sources_match_host(backend):
    shape, delta = (24, 20, 28), 1.0 / 24.0
    rng0 = np.random.default_rng(3)
    n0 = 4000
    pos = (rng0.random((n0, 3)) * np.asarray(shape) * delta).astype(np.float32)
    vel = rng0.standard_normal((n0, 3)).astype(np.float32)
    inflow = box_mask(shape, (2, 12, 3), (7, 18, 9))
    inflow2 = box_mask(shape, (15, 2, 15), (20, 6, 22))
    outflow = box_mask(shape, (10, 0, 0), (14, 5, 28))
    obstacle = box_mask(shape, (4, 14, 4), (5, 15, 6))
    host_sources = [{"type": "OUTFLOW", "mask": outflow.astype(bool)},
                    {"type": "INFLOW", "mask": inflow.astype(bool), "particle_density": 8, "velocity": (0.0, -1.5, 0.25)},
                    {"type": "INFLOW", "mask": inflow2.astype(bool), "particle_density": 5, "velocity": (0.5, 0.0, 0.0)}]
    dev = "cuda"
    dev_sources = [{"type": s["type"], "mask_device": torch.from_numpy(s["mask"].astype(np.uint8)).to(dev),
                    **{k: v for k, v in s.items() if k not in ("type", "mask")}} for s in host_sources]
    sim = solver.FlipSolver(backend, shape, delta, pos, vel, capacity=n0)
    rng_h, rng_d = np.random.default_rng(11), np.random.default_rng(11)
    ds = source_particles.DeviceSources(backend, dev_sources, torch.from_numpy(obstacle).to(dev), shape, delta, rng_d)
    hp, hv = pos.copy(), vel.copy()
    for rnd in range(4):
        hp, hv = host_sources_oracle.apply_sources(hp, hv, host_sources, obstacle.astype(bool), delta, rng_h)
        ds.apply(sim)
        assert sim.n == len(hp), rnd
        assert np.array_equal(sim.positions(), hp), rnd
        assert np.array_equal(sim.velocities(), hv), rnd
        # move every particle the same way on both sides so the next round has work to do
        shift = np.float32(0.37 * delta)
        hp = np.mod(hp + shift, np.float32(shape[0] * delta * 0.9)).astype(np.float32)
        sim.particles[: sim.n].copy_(torch.from_numpy(hp).to(dev))
    assert sim.particles.shape[0] > n0  # the buffers grew
    assert rng_d.random() == rng_h.random()  # the generator continues where the host's does
    assert backend.device_error() == 0


def test_initial_fill_matches_host(backend):
    """apply_sources(initial=True): geometry sources and inflows filled in their order into an
    empty scene (overlapping sources top each other up), as solver.py:146-158 seeds a bake."""
    shape, delta = (20, 24, 18), 1.0 / 20.0
    pool = box_mask(shape, (1, 1, 1), (19, 23, 6))
    ball = box_mask(shape, (6, 8, 4), (12, 14, 10))
    inflow = box_mask(shape, (2, 2, 12), (5, 5, 15))
    obstacle = box_mask(shape, (8, 10, 2), (10, 12, 4))
    host = [{"type": "GEOMETRY", "mask": pool.astype(bool), "particle_density": 8},
            {"type": "GEOMETRY", "mask": ball.astype(bool), "particle_density": 8, "velocity": (0.0, 0.0, -2.0)},
            {"type": "INFLOW", "mask": inflow.astype(bool), "particle_density": 6, "velocity": (1.0, 0.0, 0.0)}]
    dev = [{"type": s["type"], "mask_device": torch.from_numpy(s["mask"].astype(np.uint8)).to("cuda"),
            **{k: v for k, v in s.items() if k not in ("type", "mask")}} for s in host]
    empty = np.zeros((0, 3), np.float32)
    sim = solver.FlipSolver(backend, shape, delta, empty, empty)
    rng_h, rng_d = np.random.default_rng(0), np.random.default_rng(0)
    source_particles.DeviceSources(backend, dev, torch.from_numpy(obstacle).to("cuda"), shape, delta, rng_d,
                                   initial=True).apply(sim)
    hp, hv = host_sources_oracle.apply_sources(empty, empty, host, obstacle.astype(bool), delta, rng_h, initial=True)
    assert sim.n == len(hp) > 0
    assert np.array_equal(sim.positions(), hp) and np.array_equal(sim.velocities(), hv)
    assert rng_d.random() == rng_h.random()
    assert backend.device_error() == 0
