"""The tiled P2G (each particle visited once, the tolerance-mode path) against the reference-order
gather and the oracle: the fluid fraction bit for bit, the face velocities within 1e-5 of the field's
largest magnitude (only the order and rounding of each cell's sums differ, so a sum that cancels can
come out as an exact 0 in one order and a tiny value in the other), the same bits on every run; at 64^3 and at
the 256^3 block of the benchmark."""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-5


def bin_and_gather(backend, pos, vel, shape, dx, tiled):
    from continuum_liquid_b200 import particles as pm

    n = len(pos)
    dev = backend.device
    p = torch.from_numpy(np.ascontiguousarray(pos, np.float32)).to(dev)
    v = torch.from_numpy(np.ascontiguousarray(vel, np.float32)).to(dev)
    work, vwork, counts, outputs, sums = pm.create_particle_sort_buffers(backend, shape, n)
    grid = [torch.zeros(shape, dtype=torch.float32, device=dev) for _ in range(4)]
    pm.particle_to_grid(backend, None, p, v, work, vwork, tuple(grid[:3]), counts, outputs, sums, grid[3], n, shape,
                        dx, 8, tiled=tiled)
    return [g.cpu().numpy() for g in grid[:3]], grid[3].cpu().numpy()


def check_close(got, ref):
    for a, b in zip(got, ref):
        scale = float(np.abs(b).max()) or 1.0
        assert float(np.abs(a.astype(np.float64) - b).max()) <= TOL * scale


def scene_particles(kind, n):
    from continuum_liquid_b200 import scenes

    if kind == "block":
        s = scenes.block(n)
    elif kind == "dam":
        s = scenes.dam_break(n, seed=1)
    else:
        s = scenes.collider_pool(n, seed=1, subdivisions=2)
    pos, _ = scenes.seed_particles(s)
    rng = np.random.default_rng(7)
    vel = rng.standard_normal(pos.shape).astype(np.float32)
    return s, pos, vel


@pytest.mark.parametrize("kind,n", [("dam", 37), ("pool", 48), ("dam", 64)])
def test_tiled_p2g_matches_gather_and_oracle(backend, oracle, kind, n):
    s, pos, vel = scene_particles(kind, n)
    exact, ff_e = bin_and_gather(backend, pos, vel, s.grid_shape, s.dx, tiled=False)
    tiled, ff_t = bin_and_gather(backend, pos, vel, s.grid_shape, s.dx, tiled=True)
    again, ff_a = bin_and_gather(backend, pos, vel, s.grid_shape, s.dx, tiled=True)
    assert np.array_equal(ff_t, ff_e)
    check_close(tiled, exact)
    assert all(np.array_equal(a, b) for a, b in zip(tiled, again)) and np.array_equal(ff_a, ff_t)
    _, _, u, v, w, ff, _, _ = oracle.particle_to_grid(pos, vel, s.dx, s.grid_shape)
    assert np.array_equal(ff_t, ff)
    check_close(tiled, (u, v, w))
    assert backend.device_error() == 0


def test_tiled_p2g_dense_and_empty_bins(backend, oracle):
    """Particles piled into a few bins (hundreds per bin) next to empty tiles."""
    shape, dx = (44, 31, 70), 1.0 / 64
    rng = np.random.default_rng(3)
    centres = np.array([[5.5, 7.2, 9.9], [20.1, 15.5, 33.3], [40.0, 28.0, 66.0]]) * dx
    pos = np.concatenate([c + rng.normal(0, 0.6 * dx, (3000, 3)) for c in centres]).astype(np.float32)
    pos = np.clip(pos, 1.001 * dx, (np.array(shape) - 1.001) * dx).astype(np.float32)
    vel = rng.standard_normal(pos.shape).astype(np.float32)
    tiled, ff_t = bin_and_gather(backend, pos, vel, shape, dx, tiled=True)
    _, _, u, v, w, ff, _, _ = oracle.particle_to_grid(pos, vel, dx, shape)
    assert np.array_equal(ff_t, ff)
    check_close(tiled, (u, v, w))


def test_tiled_p2g_block_256(backend):
    """The benchmark's 256^3 block (23M particles): tiled against the reference-order gather on the
    GPU, which the oracle pins bit for bit (bench.py's parity object checks that one)."""
    s, pos, vel = scene_particles("block", 256)
    exact, ff_e = bin_and_gather(backend, pos, vel, s.grid_shape, s.dx, tiled=False)
    torch.cuda.empty_cache()
    tiled, ff_t = bin_and_gather(backend, pos, vel, s.grid_shape, s.dx, tiled=True)
    assert np.array_equal(ff_t, ff_e)
    check_close(tiled, exact)
    assert backend.device_error() == 0
