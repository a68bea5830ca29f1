"""Batched scenes: one launch per stage for scenes of different sizes (continuum_liquid_b200/batch.py).

Reference mode (fixed W-cycles): every scene of the batch equals its single-scene run bit for bit,
with and without CUDA graphs. Tolerance mode: every scene reaches the tolerance."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from continuum_liquid_b200 import batch, scenes, solver

pytestmark = pytest.mark.gpu


def mixed_scenes():
    # pyramids: 16 -> (16, 9) and 20 -> (20, 11) end in a coarse solve; 24 and 32 end in a bottom visit
    return [scenes.dam_break(16, seed=1), scenes.collider_pool(20, seed=2, subdivisions=2),
            scenes.block(24, seed=3), scenes.collider_pool(32, seed=5, subdivisions=2)]


def single(backend, sc, **kw):
    opts = solver.StepOptions(flip_ratio=0.95, gravity=sc.gravity, rho=sc.rho, nu=sc.nu, use_graph=False, **kw)
    return solver.scene_solver(backend, sc, opts)


def test_bottom_plan_matches_the_library_rule():
    assert batch.bottom_plan([(16, 16, 16), (9, 9, 9)])[0] == -1
    assert batch.bottom_plan([(32, 32, 32), (17, 17, 17), (10, 10, 10)])[0] == 1
    assert batch.bottom_plan([(160,) * 3, (81,) * 3, (42,) * 3, (22,) * 3, (12,) * 3])[0] == -1  # 22^3 too large


@pytest.mark.parametrize("use_graph", [True, False])
def test_reference_mode_matches_single_scenes(backend, use_graph):
    sc = mixed_scenes()
    b = batch.BatchedFlip(backend, sc, flip_ratio=0.95, tol=None, num_vcycles=1, use_graph=use_graph)
    assert [p[0] for p in b.plans] == [-1, -1, 1, 1]
    sims = [single(backend, s, num_vcycles=1) for s in sc]
    for s, sim in enumerate(sims):
        assert np.array_equal(b.positions(s), sim.positions())
        assert np.array_equal(b.scene_view(b.obstacle, s).cpu().numpy(),
                              (sim.obstacle if sim.obstacle is not None else
                               torch.zeros(sim.grid_shape, dtype=torch.uint8)).cpu().numpy())
    for step in range(3):
        b.step()
        for s, sim in enumerate(sims):
            sim.step()
            host = lambda t: t.detach().cpu().numpy()  # noqa: E731
            assert np.array_equal(host(b.scene_view(b.pressure, s)), host(sim.pressure)), (step, s, "pressure")
            for got, want, name in ((b.u, sim.u, "u"), (b.v, sim.v, "v"), (b.w, sim.w, "w")):
                assert np.array_equal(host(b.scene_view(got, s)), host(want)), (step, s, name)
            assert np.array_equal(b.positions(s), sim.positions()), (step, s, "positions")
            assert np.array_equal(b.velocities(s), sim.velocities()), (step, s, "velocities")
    assert backend.device_error() == 0


@pytest.mark.parametrize("wset", [{}, {"coarse_iterations": 4, "pre_smooth": 1, "post_smooth": 1},
                                  {"coarse_iterations": 0, "pre_smooth": 1, "post_smooth": 1, "prolong_scale": 1.7},
                                  {"coarse_iterations": 0, "pre_smooth": 1, "post_smooth": 1, "prolong_scale": 1.8,
                                   "coarse_smooth": (1, 0)}],
                         ids=["reference-cycle", "c4-s11", "c0-s11-w17", "c0-s11-w18-cs10"])
def test_tolerance_mode_solves_every_scene(backend, wset):
    sc = mixed_scenes()
    b = batch.BatchedFlip(backend, sc, flip_ratio=0.95, tol=1e-6, **wset)
    sims = [single(backend, s, tol=1e-6, **wset) for s in sc]
    for step in range(4):
        st = b.step()
        assert len(st.rel_residual) == len(sc) and max(st.rel_residual) <= 1e-6
        for s, sim in enumerate(sims):
            sim.step()
            # the batch iterates until its slowest scene converges, so scenes agree within the tolerance
            diff = np.abs(b.positions(s) - sim.positions()).max()
            assert diff <= 1e-5 * sc[s].grid_shape[0] * sc[s].dx, (step, s, diff)
    assert b.graph_replays > 0
    assert backend.device_error() == 0


@pytest.mark.parametrize("tiled", [True, False])
def test_batched_p2g_matches_single_scenes(backend, tiled):
    """The batch's P2G (the tiled scatter in tolerance mode, the reference-order gather otherwise) gives
    each scene exactly the single-scene P2G's grid: the stages up to the pressure solve, bit for bit."""
    sc = mixed_scenes()
    b = batch.BatchedFlip(backend, sc, flip_ratio=0.95, tol=1e-6 if tiled else None, use_graph=False)
    assert b.batch.p2g_tiled == int(tiled)
    sims = [single(backend, s, tol=1e-6 if tiled else None) for s in sc]
    assert all(sim.options.tiled_p2g() == tiled for sim in sims)
    b.pre_solve()
    host = lambda t: t.detach().cpu().numpy()  # noqa: E731
    for s, sim in enumerate(sims):
        sim.pre_solve()
        for got, want, name in ((b.u, sim.u, "u"), (b.v, sim.v, "v"), (b.w, sim.w, "w"),
                                (b.fluid_fraction, sim.fluid_fraction, "fluid fraction")):
            assert np.array_equal(host(b.scene_view(got, s)), host(want)), (s, name)
    assert backend.device_error() == 0
