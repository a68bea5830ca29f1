"""Parity against the reference solver itself.

The fixtures tests/golden/ref_* were produced by running the reference's own main(config) (its
Python host code and its OpenCL kernels, on the CPU through oracle/reference_run.py) on the bakes of
tests/golden/reference_scenes.py; tests/golden/make_reference_golden.py is the recipe.

CPU (always): the oracle's restated bake reproduces every stored frame, mask and first-step
intermediate bit for bit (value equality; -0 equals +0); the large scenes are compared through the
stored digests for their first frames. When the reference checkout is present, the recipe itself is
re-run on the smallest scene and must reproduce its fixture.

GPU: this backend's drop-in entry point `general.main(config)` bakes the same configs and writes
the same particle cache, frame for frame, bit for bit: the three small scenes, the 64^3 dam break
for all 120 steps, the 128^3 collider pool (its 5120-triangle collider voxelised by the CUDA
kernel) and the first step of the 256^3 block, whose intermediates (per-cell counts, offsets,
sorted order, P2G, pressure, projected velocity) are checked against the reference's digests too.
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))

import reference_scenes as rs  # noqa: E402

ORACLE_KEYS = {"pos_sorted": "sorted_pos", "vel_sorted": "sorted_vel"}
STEP_KEYS = ("counts", "offsets", "pos_sorted", "vel_sorted", "p2g_u", "p2g_v", "p2g_w", "p2g_ff", "pre_u", "pre_v",
             "pre_w", "ff", "pressure_in", "rhs", "pressure", "vel_g2p", "u", "v", "w")


def load_small(name):
    with np.load(GOLDEN / f"ref_{name}.npz") as d:
        data = {k: d[k] for k in d.files}
    return json.loads(str(data.pop("meta"))), data


def load_large(name):
    return json.loads((GOLDEN / f"ref_{name}.json").read_text())


def equal(a, b) -> bool:
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a, b)


@pytest.mark.parametrize("name", rs.SMALL + rs.LARGE)
def test_fixture_matches_scene_definition(name):
    meta = load_small(name)[0] if name in rs.SMALL else load_large(name)
    assert meta["config_digest"] == rs.config_digest(rs.scene(name))


@pytest.mark.parametrize("name", rs.SMALL)
def test_oracle_bake_reproduces_reference(oracle, name):
    from oracle import bake

    meta, ref = load_small(name)
    out = bake.bake(rs.scene(name))
    for key, mask in out["masks"].items():
        assert equal(mask, ref[f"mask_{key}"]), key
    assert len(out["frames"]) == len(meta["frames"])
    for i, (frame, info) in enumerate(zip(out["frames"], meta["frames"])):
        assert rs.digest(frame) == info["digest"], f"frame {i}"
        if f"frame_{i:03d}" in ref:
            assert equal(frame, ref[f"frame_{i:03d}"]), f"frame {i}"
    step = out["steps"][0]
    for key in STEP_KEYS:
        got = step[ORACLE_KEYS.get(key, key)]
        assert equal(np.asarray(got).reshape(ref[f"s1_{key}"].shape), ref[f"s1_{key}"]), key


def test_oracle_bake_reproduces_reference_dam_break_64(oracle):
    """The 64^3 dam break (120 reference steps stored): the oracle's first 5 frames and every
    intermediate of its first step equal the reference's (the GPU test runs all 120)."""
    from oracle import bake

    meta = load_large("config1_dam_break_64")
    out = bake.bake(rs.scene("config1_dam_break_64"), max_frames=5)
    for i, frame in enumerate(out["frames"]):
        assert rs.digest(frame) == meta["frames"][i]["digest"], f"frame {i}"
    step = out["steps"][0]
    for key in STEP_KEYS:
        got = np.asarray(step[ORACLE_KEYS.get(key, key)])
        if key in ("counts", "offsets", "p2g_u", "p2g_v", "p2g_w", "p2g_ff", "pre_u", "pre_v", "pre_w", "ff",
                   "pressure_in", "rhs", "pressure", "u", "v", "w"):
            got = got.reshape(out["grid_shape"])
        assert rs.digest(got) == meta["step1"][key], key


def test_oracle_voxelises_config2_collider(oracle):
    """The 128^3 collider of 5120 triangles: the oracle's ray-parity voxelisation equals the
    reference's mask bit for bit."""
    from oracle import bake

    cfg = rs.scene("config2_collider_pool_128")
    sim = cfg["simulation"]
    delta = sim["domain"]["resolution"]
    entries = [e for o in sim["obstacles"] for e in o["geometry_inputs"]]
    assert sum(len(e["triangles"]) for e in entries) == 5120
    mask = bake.voxelise_entries(entries, (128, 128, 128), delta, (-0.5, -0.5, 0.0))
    with np.load(GOLDEN / "ref_config2_collider_pool_128_obstacle.npz") as d:
        ref = np.unpackbits(d["bits"])[: int(np.prod(d["shape"]))].reshape(tuple(d["shape"]))
    assert mask.any() and equal(mask, ref)
    assert rs.digest(mask) == load_large("config2_collider_pool_128")["masks"]["obstacle"]


def test_reference_recipe_reproduces_fixture():
    """Re-runs the reference itself (when its checkout is here) on the 16^3 dam break."""
    from oracle import reference_run

    if not reference_run.available():
        pytest.skip("reference checkout not present")
    meta, ref = load_small("dam_break_16")
    cfg = rs.scene("dam_break_16")
    record = reference_run.run(cfg, rs.meshes(cfg))
    assert [rs.digest(f) for f in record["frames"]] == [f["digest"] for f in meta["frames"]]
    for key in STEP_KEYS:
        assert equal(record["steps"][0][key], ref[f"s1_{key}"]), key


# ---- GPU: the drop-in entry point against the reference's bakes --------------------------------
def bake_with_backend(name, tmp_path):
    from continuum_liquid_b200.general import main as general

    cfg = rs.scene(name)
    cfg["simulation"] = dict(cfg["simulation"], output_path=str(tmp_path / name))
    messages = []
    general.set_message_callback(messages.append)
    try:
        general.main(cfg)
    finally:
        general.clear_message_callback()
    frames = sorted((tmp_path / name / "particles").glob("particles_*.bin"))
    return [np.fromfile(f, dtype=np.float32).reshape(-1, 3) for f in frames], messages


@pytest.mark.gpu
@pytest.mark.parametrize("name", rs.SMALL + ("config1_dam_break_64", "config2_collider_pool_128"))
def test_main_bakes_the_reference_cache(backend, tmp_path, name):
    meta = load_small(name)[0] if name in rs.SMALL else load_large(name)
    frames, messages = bake_with_backend(name, tmp_path)
    assert len(frames) == len(meta["frames"])
    for i, (frame, info) in enumerate(zip(frames, meta["frames"])):
        assert len(frame) == info["count"], f"frame {i}"
        assert rs.digest(frame) == info["digest"], f"frame {i}"
    stats = [m for m in messages if m.get("type") == "stats"]
    assert [m["particle_count"] for m in stats] == [m["particle_count"] for m in meta["messages"]]
    assert backend.device_error() == 0


@pytest.mark.gpu
def test_block_256_first_step_matches_reference(backend):
    """The 256^3 block (23M particles): seeding on the device, then the first step through the stage
    API in reference mode; every intermediate's digest equals the reference's."""
    import torch

    from continuum_liquid_b200 import boundary_conditions, particles as pm, solver, source_particles
    from continuum_liquid_b200 import velocity_update, voxelise_mesh

    meta = load_large("config3_block_256")
    cfg = rs.scene("config3_block_256")
    sim_cfg = cfg["simulation"]
    shape, delta, dt = (256, 256, 256), 1.0 / 256, 1.0 / 240
    sources_dev, obstacle = voxelise_mesh.build_static_masks(backend, None, backend, sim_cfg, shape, delta)
    for i, src in enumerate(sources_dev):
        assert rs.digest(src["mask_device"].cpu().numpy()) == meta["masks"][f"source{i}"]
    sim = solver.FlipSolver(backend, shape, delta, np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32),
                            dt=dt, options=solver.StepOptions(use_graph=False))
    seeder = source_particles.DeviceSources(backend, sources_dev, None, shape, delta, np.random.default_rng(0),
                                            initial=True)
    seeder.apply(sim)
    assert sim.n == meta["frames"][0]["count"]
    assert rs.digest(sim.positions()) == meta["frames"][0]["digest"]
    host = lambda t: t.detach().cpu().numpy()  # noqa: E731
    k, n = backend, sim.n
    (sim.particles, sim.particle_velocity, sim.particle_work, sim.particle_velocity_work, _,
     sim.fluid_fraction) = pm.particle_to_grid(k, None, sim.particles, sim.particle_velocity, sim.particle_work,
                                               sim.particle_velocity_work, (sim.u, sim.v, sim.w), sim.bin_counts,
                                               sim.scan_outputs, sim.scan_sums, sim.fluid_fraction, n, shape,
                                               delta, 8)
    got = {"counts": host(sim.bin_counts).reshape(shape), "offsets": host(sim.scan_outputs[0]).reshape(shape),
           "pos_sorted": sim.positions(), "vel_sorted": sim.velocities(), "p2g_u": host(sim.u), "p2g_v": host(sim.v),
           "p2g_w": host(sim.w), "p2g_ff": host(sim.fluid_fraction)}
    vel = (sim.u, sim.v, sim.w)
    boundary_conditions.grid_domain_bc(k, None, vel, shape)
    velocity_update.update_velocity(k, None, vel, (sim.u_work, sim.v_work, sim.w_work), sim.fluid_fraction,
                                    (0.0, 0.0, -9.81), 0.0, 0.0, 0.0, 1000.0, 1e-6, delta, dt, shape)
    sim.u, sim.u_work = sim.u_work, sim.u
    sim.v, sim.v_work = sim.v_work, sim.v
    sim.w, sim.w_work = sim.w_work, sim.w
    boundary_conditions.grid_domain_bc(k, None, (sim.u, sim.v, sim.w), shape)
    got.update(pre_u=host(sim.u), pre_v=host(sim.v), pre_w=host(sim.w), ff=host(sim.fluid_fraction),
               pressure_in=host(sim.pressure))
    sim.solve()
    got.update(pressure=host(sim.pressure), rhs=host(sim.pressure_solver.rhs))
    sim.post_solve()
    got.update(u=host(sim.u), v=host(sim.v), w=host(sim.w))
    for key, value in got.items():
        assert rs.digest(value) == meta["step1"][key], key
    assert rs.digest(sim.positions()) == meta["frames"][1]["digest"]
    assert backend.device_error() == 0
    del torch
