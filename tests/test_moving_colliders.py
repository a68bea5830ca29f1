"""Moving colliders (no counterpart in the reference, whose colliders never move): the rigid motion's
pose and velocity, the oracle's moving obstacle conditions at rest against the reference restatement,
and a moving paddle that pushes still liquid; on the GPU the CUDA path against the oracle, bit for bit,
and the drop-in entry with a moving obstacle in its config."""

from __future__ import annotations

import numpy as np
import pytest

from continuum_liquid_b200 import scenes
from continuum_liquid_b200.colliders import RigidMotion

MOTION = RigidMotion(velocity=(0.6, 0.0, -0.3), angular_velocity=(0.0, 4.0, 1.5), pivot=(-0.2, -0.35, 0.1))


def paddle_scene(n=24):
    """A pool with a box paddle, moving as MOTION; gravity along -y as the benchmark scenes."""
    s = scenes.Scene(f"paddle_{n}", (n, n, n), 1.0 / n, [scenes.Source(scenes.box((0, 0, 0), (1, 0.35, 1)))],
                     steps=10, seed=5)
    lo, hi = np.array([-0.3, -0.45, 0.0]), np.array([-0.1, -0.25, 0.2])
    from tests.golden.reference_scenes import box_triangles  # noqa: E402

    s.obstacles = [box_triangles(lo, hi)]
    return s


def test_rigid_motion_pose_and_velocity():
    tris = scenes.icosphere(1, 0.1, (0.05, -0.02, 0.3))
    assert np.array_equal(MOTION.transform(tris, 0.0), tris)
    # a full turn about the axis brings the mesh back, moved by V t
    period = 2 * np.pi / np.linalg.norm(MOTION.angular_velocity)
    back = MOTION.transform(tris, period) - np.asarray(MOTION.velocity, np.float32) * np.float32(period)
    assert np.allclose(back, tris, atol=1e-5)
    # the velocity field V + W x (x - C(t)) is the time derivative of the pose
    t, h = 0.3, 1e-6
    x = MOTION.transform(tris, t).astype(np.float64)
    deriv = (MOTION.transform(tris, t + h).astype(np.float64) - MOTION.transform(tris, t - h).astype(np.float64)) / (2 * h)
    want = np.asarray(MOTION.velocity) + np.cross(np.asarray(MOTION.angular_velocity), x - MOTION.pivot_at(t))
    assert np.allclose(deriv, want, atol=2e-2)
    p = MOTION.parameters(t, (-0.5, -0.5, 0.0))
    assert p.dtype == np.float32 and np.allclose(p[6:], MOTION.pivot_at(t) - np.array([-0.5, -0.5, 0.0]))


def rest_pose(scene):
    return lambda t: (scene.obstacles, np.zeros(9, np.float32))


def moving_pose(scene, motion):
    return lambda t: ([motion.transform(tri, t) for tri in scene.obstacles], motion.parameters(t, scene.origin))


def test_oracle_moving_conditions_at_rest_equal_the_reference(oracle):
    s = paddle_scene(20)
    mask = np.zeros(s.grid_shape, np.uint8)
    for tri in s.obstacles:
        mask = oracle.voxelise(tri, s.grid_shape, s.dx, s.origin, mask)
    pos, vel = scenes.seed_particles(s, mask)
    vel = np.random.default_rng(1).standard_normal(pos.shape).astype(np.float32)
    static = oracle.OracleSim(s.grid_shape, s.dx, pos, vel, obstacle=mask, dt=s.dt, flip_ratio=0.95,
                              gravity=s.gravity)
    rest = oracle.OracleSim(s.grid_shape, s.dx, pos, vel, obstacle=mask, dt=s.dt, flip_ratio=0.95, gravity=s.gravity,
                            collider_pose=rest_pose(s), origin=s.origin)
    for _ in range(3):
        static.step()
        rest.step()
    assert np.array_equal(static.pos, rest.pos) and np.array_equal(static.vel, rest.vel)


def test_moving_paddle_pushes_still_liquid(oracle):
    """No gravity, liquid at rest: a paddle moving along +x gives the liquid +x momentum."""
    s = paddle_scene(20)
    motion = RigidMotion(velocity=(1.0, 0.0, 0.0), pivot=(-0.2, -0.35, 0.1))
    mask = np.zeros(s.grid_shape, np.uint8)
    for tri in s.obstacles:
        mask = oracle.voxelise(tri, s.grid_shape, s.dx, s.origin, mask)
    pos, vel = scenes.seed_particles(s, mask)
    sim = oracle.OracleSim(s.grid_shape, s.dx, pos, vel, obstacle=mask, dt=s.dt, flip_ratio=0.95,
                           gravity=(0.0, 0.0, 0.0), collider_pose=moving_pose(s, motion), origin=s.origin)
    for _ in range(6):
        sim.step()
    assert sim.vel[:, 0].mean() > 1e-3
    assert abs(sim.vel[:, 2].mean()) < 0.2 * sim.vel[:, 0].mean()


@pytest.mark.gpu
@pytest.mark.parametrize("motion", [MOTION, RigidMotion()])
def test_cuda_moving_collider_matches_oracle(backend, oracle, motion):
    import torch

    from continuum_liquid_b200 import solver, voxelise_mesh

    s = paddle_scene(24)
    mask = torch.zeros(s.grid_shape, dtype=torch.uint8, device="cuda")
    for tri in s.obstacles:
        voxelise_mesh.voxelise_triangles(backend, None, tri, mask, s.grid_shape, s.dx, s.origin)
    pos, vel = scenes.seed_particles(s, mask.cpu().numpy())
    opts = solver.StepOptions(flip_ratio=0.95, num_vcycles=1, gravity=s.gravity, use_graph=False)
    sim = solver.FlipSolver(backend, s.grid_shape, s.dx, pos, vel, obstacle=mask, dt=s.dt, options=opts,
                            colliders=s.obstacles, origin=s.origin, collider_motion=motion)
    ref = oracle.OracleSim(s.grid_shape, s.dx, pos, vel, obstacle=mask.cpu().numpy(), dt=s.dt, flip_ratio=0.95,
                           gravity=s.gravity, collider_pose=moving_pose(s, motion), origin=s.origin)
    for step in range(5):
        sim.step()
        ref.step()
        assert np.array_equal(sim.obstacle.cpu().numpy(), ref.obstacle), f"obstacle, step {step}"
        assert np.array_equal(sim.positions(), ref.pos), f"positions, step {step}"
        assert np.array_equal(sim.velocities(), ref.vel), f"velocities, step {step}"
    if motion == RigidMotion():  # at rest: the static path's results
        static = solver.FlipSolver(backend, s.grid_shape, s.dx, pos, vel, obstacle=mask, dt=s.dt, options=opts)
        for _ in range(5):
            static.step()
        assert np.array_equal(static.positions(), sim.positions())
    assert backend.device_error() == 0


@pytest.mark.gpu
def test_main_with_a_moving_obstacle(backend, tmp_path):
    from continuum_liquid_b200.general import main as general
    from tests.golden.reference_scenes import box_triangles, config, entry

    cfg = config(24, 4, [{"type": "GEOMETRY", "particle_density": 8,
                          "geometry_inputs": [entry("pool", box_triangles((-0.5, -0.5, 0.0), (0.5, 0.5, 0.3)))]}],
                 [entry("paddle", box_triangles((-0.3, -0.1, 0.0), (-0.1, 0.1, 0.4)))])
    cfg["simulation"]["obstacles"][0]["motion"] = {"velocity": [0.8, 0.0, 0.0], "pivot": [-0.2, 0.0, 0.2]}
    cfg["simulation"]["output_path"] = str(tmp_path / "bake")
    general.main(cfg)
    frames = sorted((tmp_path / "bake" / "particles").glob("particles_*.bin"))
    assert len(frames) == 5
    last = np.fromfile(frames[-1], dtype=np.float32).reshape(-1, 3)
    assert np.isfinite(last).all() and len(last) > 0
    bad = dict(cfg)
    bad["simulation"] = dict(cfg["simulation"], obstacles=[cfg["simulation"]["obstacles"][0],
                                                            {"geometry_inputs": [entry("post", box_triangles(
                                                                (0.2, 0.2, 0.0), (0.3, 0.3, 0.5)))]}])
    with pytest.raises(ValueError, match="same motion"):
        general.main(bad)
