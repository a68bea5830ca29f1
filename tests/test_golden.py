"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py from the oracle).

CPU: the scene generator reproduces the stored inputs and the oracle reproduces every stored value
bit for bit. GPU: the CUDA backend, driven through the stage API in reference mode (pure FLIP or the
stored blend, one W-cycle per step), reproduces them bit for bit as well."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
NAMES = ["dam_break_16", "collider_pool_16"]
TRACE = ("counts", "offsets", "sorted_pos", "p2g_u", "p2g_ff", "rhs", "pressure", "u", "v", "w")


def load(name):
    with np.load(GOLDEN / f"{name}.npz") as d:
        return {k: d[k] for k in d.files}


@pytest.mark.parametrize("name", NAMES)
def test_scene_generator_reproduces_inputs(oracle, name):
    import sys

    sys.path.insert(0, str(GOLDEN))
    from make_golden import CASES

    from continuum_liquid_b200 import scenes

    g = load(name)
    s = CASES[name][0](scenes)
    assert tuple(g["grid_shape"]) == s.grid_shape
    tris = np.concatenate([np.asarray(t, np.float32) for t in s.obstacles]) if s.obstacles else \
        np.zeros((0, 3, 3), np.float32)
    assert np.array_equal(tris, g["triangles"])
    assert np.array_equal(oracle.voxelise(tris, s.grid_shape, s.dx, s.origin), g["obstacle"]) if len(tris) else True
    pos, vel = scenes.seed_particles(s, g["obstacle"])
    assert np.array_equal(pos, g["in_pos"]) and np.array_equal(vel, g["in_vel"])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_fixture(oracle, name):
    g = load(name)
    shape = tuple(int(x) for x in g["grid_shape"])
    sim = oracle.OracleSim(shape, float(g["dx"]), g["in_pos"], g["in_vel"], obstacle=g["obstacle"],
                           dt=float(g["dt"]), flip_ratio=float(g["flip_ratio"]), gravity=tuple(g["gravity"]))
    for _ in range(int(g["steps"])):
        sim.step()
    for key in TRACE:
        assert np.array_equal(sim.trace[key], g[key]), key
    assert np.array_equal(sim.pos, g["out_pos"]) and np.array_equal(sim.vel, g["out_vel"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_cuda_backend_reproduces_fixture(backend, name):
    import torch

    from continuum_liquid_b200 import solver, voxelise_mesh

    g = load(name)
    shape = tuple(int(x) for x in g["grid_shape"])
    dx = float(g["dx"])
    mask = torch.zeros(shape, dtype=torch.uint8, device="cuda")
    if len(g["triangles"]):
        voxelise_mesh.voxelise_triangles(backend, None, g["triangles"], mask, shape, dx, tuple(g["origin"]))
    assert np.array_equal(mask.cpu().numpy(), g["obstacle"])
    opts = solver.StepOptions(flip_ratio=float(g["flip_ratio"]), num_vcycles=1, gravity=tuple(g["gravity"]),
                              use_graph=False)
    sim = solver.FlipSolver(backend, shape, dx, g["in_pos"], g["in_vel"], obstacle=g["obstacle"], dt=float(g["dt"]),
                            options=opts)
    for _ in range(int(g["steps"])):
        sim.step()
    host = lambda t: t.detach().cpu().numpy()  # noqa: E731
    assert np.array_equal(host(sim.bin_counts), g["counts"])
    assert np.array_equal(host(sim.pressure), g["pressure"])
    for got, key in ((sim.u, "u"), (sim.v, "v"), (sim.w, "w")):
        assert np.array_equal(host(got), g[key]), key
    assert np.array_equal(sim.positions(), g["out_pos"]) and np.array_equal(sim.velocities(), g["out_vel"])
    assert backend.device_error() == 0
