"""The tolerance-mode iteration looping on the device (clb_solve_loop_*: a CUDA graph with a WHILE
conditional node) against the host loop: the same refinements, so the same residual history cycle for
cycle and the same FP64 pressure when both stop after the same refinement; the loop stops at the first
refinement that meets the tolerance, and at max_cycles."""

import numpy as np
import pytest
import torch

from continuum_liquid_b200 import pressure_solve, scenes, solver

pytestmark = pytest.mark.gpu


def run_steps(backend, device_loop, steps, **kw):
    s = scenes.block(48, seed=3)
    opts = solver.StepOptions(flip_ratio=0.95, tol=1e-6, gravity=s.gravity, coarse_iterations=4, pre_smooth=1,
                              post_smooth=1)
    pos, vel = scenes.seed_particles(s)
    sim = solver.FlipSolver(backend, s.grid_shape, s.dx, pos, vel, dt=s.dt, options=opts, min_size=s.min_size)
    sim.pressure_solver = pressure_solve.PressureSolver(backend, s.grid_shape, s.dx, min_size=s.min_size,
                                                        coarse_iterations=4, pre_smooth=1, post_smooth=1,
                                                        device_loop=device_loop, **kw)
    sim.pressure_solver.host_batch = 1  # the host loop reads the residual after every refinement
    out = []
    for _ in range(steps):
        st = sim.step()
        out.append((st.cycles, list(st.history), sim.pressure_solver.pressure64.cpu().numpy().copy()))
    return sim, out


@pytest.mark.parametrize("method", ["fcg", "refine"])
def test_device_loop_matches_host_loop(backend, method):
    sim_d, dev = run_steps(backend, True, 5, method=method)
    sim_h, host = run_steps(backend, False, 5, method=method)
    assert sim_d.pressure_solver._loop is not None, getattr(sim_d.pressure_solver, "loop_error", "")
    assert sim_d.pressure_solver.loop_refinements > 0
    assert sim_h.pressure_solver.loop_refinements == 0
    for (cd, hd, pd), (ch, hh, ph) in zip(dev, host):
        # the device loop stops at the first refinement at or below the tolerance
        first = next(k for k, r in enumerate(hh) if r <= 1e-6)
        assert cd == first, (cd, first, hh)
        assert hd == hh[: cd + 1]  # the same refinements: the same residuals, bit for bit
        assert hd[-1] <= 1e-6
        assert cd == ch  # with a read after every refinement the host loop stops there too
        assert np.array_equal(pd, ph)
    assert backend.device_error() == 0


def test_device_loop_stops_at_max_cycles(backend):
    sim, out = run_steps(backend, True, 4, max_cycles=3)
    for cycles, hist, _ in out[1:]:  # solves after the first run the device loop
        assert cycles == 3 and len(hist) == 4
    assert backend.device_error() == 0
