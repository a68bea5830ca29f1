"""The particle update walking the bins of tiles (clb_particle_update_tiled) against the per-particle
kernel (clb_particle_update): positions, velocities and previous positions bit for bit, with and
without an obstacle and a moving one, on grids whose bins do not fill the last tiles."""

import numpy as np
import pytest
import torch

from continuum_liquid_b200 import particles as pm
from continuum_liquid_b200 import scenes
from continuum_liquid_b200.colliders import RigidMotion

pytestmark = pytest.mark.gpu

F32 = np.float32


@pytest.mark.parametrize("case", ["dam", "pool", "pool_moving", "odd"])
def test_tiled_particle_update_matches(backend, case):
    if case == "dam":
        s = scenes.dam_break(48, seed=2)
    elif case == "odd":
        s = scenes.dam_break(37, seed=4)
        s.grid_shape = (37, 45, 71)
    else:
        s = scenes.collider_pool(40, seed=3, subdivisions=2)
    shape, dx = tuple(s.grid_shape), float(s.dx)
    dev = backend.device
    obstacle = None
    if s.obstacles:
        from continuum_liquid_b200 import voxelise_mesh

        obstacle = torch.zeros(shape, dtype=torch.uint8, device=dev)
        for tris in s.obstacles:
            voxelise_mesh.voxelise_triangles(backend, None, tris, obstacle, shape, s.dx, s.origin)
    pos, _ = scenes.seed_particles(s, None if obstacle is None else obstacle.cpu().numpy())
    pos = pos[np.all(pos < np.asarray(shape, F32) * F32(dx), axis=1)]
    rng = np.random.default_rng(5)
    vel = (rng.standard_normal(pos.shape) * 2.0).astype(F32)
    n = len(pos)
    p = torch.from_numpy(np.ascontiguousarray(pos)).to(dev)
    v = torch.from_numpy(vel).to(dev)
    work, vwork, counts, outputs, sums = pm.create_particle_sort_buffers(backend, shape, n)
    grid = [torch.zeros(shape, dtype=torch.float32, device=dev) for _ in range(4)]
    pm.particle_to_grid(backend, None, p, v, work, vwork, tuple(grid[:3]), counts, outputs, sums, grid[3], n, shape, dx,
                        8)
    # the sorted particles are in work / vwork; grid fields: random current and old velocities
    cur = [torch.from_numpy(rng.standard_normal(shape).astype(F32)).to(dev) for _ in range(3)]
    old = [torch.from_numpy(rng.standard_normal(shape).astype(F32)).to(dev) for _ in range(3)]
    motion = None
    if case == "pool_moving":
        motion = RigidMotion(velocity=(0.3, -0.2, 0.1), angular_velocity=(0.0, 1.5, 0.5),
                             pivot=(0.5, 0.3, 0.5)).parameters(0.01, s.origin)
    results = []
    for bins in (None, (outputs[0], counts)):
        pp, vv = work[:n].clone(), vwork[:n].clone()
        prev = torch.zeros_like(pp)
        pm.particle_update(backend, None, pp, vv, tuple(cur), tuple(old), obstacle, n, shape, dx, 1.0 / 240.0,
                           flip_ratio=0.95, previous_particles=prev, motion=motion, bins=bins)
        torch.cuda.synchronize()
        results.append([t.cpu().numpy() for t in (pp, vv, prev)])
    for a, b, name in zip(results[0], results[1], ("positions", "velocities", "previous")):
        assert np.array_equal(a, b), name
    assert np.abs(results[1][0] - work[:n].cpu().numpy()).max() > 0  # the particles moved
    assert backend.device_error() == 0
