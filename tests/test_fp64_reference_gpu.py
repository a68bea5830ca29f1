"""The FP64 reference solution that bench.py measures each step's pressure error against: the
FP64-accumulated flexible CG run to 1e-11 agrees with the oracle's FP64-only W-cycle solve (every
smoothing, restriction and prolongation in FP64, run to 1e-12) on the same system, so its FP32
W-cycle preconditioner changes only how fast it converges, not the answer."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["dam_break", "collider_pool"])
def test_fp64_reference_solution_matches_fp64_only_wcycle(backend, oracle, name):
    from continuum_liquid_b200 import scenes, solver
    from continuum_liquid_b200.pressure_solve import PressureSolver

    scene = scenes.dam_break(40, seed=2) if name == "dam_break" else scenes.collider_pool(40, seed=2, subdivisions=2)
    sim = solver.scene_solver(backend, scene, solver.StepOptions(flip_ratio=0.95, tol=1e-6, gravity=scene.gravity,
                                                                 rho=scene.rho, nu=scene.nu))
    sim.step()
    sim.pre_solve()
    ps = PressureSolver(backend, scene.grid_shape, scene.dx, min_size=scene.min_size, method="fcg", max_cycles=300)
    p32 = sim.pressure.clone()
    st = ps.solve((sim.u, sim.v, sim.w), sim.fluid_fraction, p32, sim.dt, scene.rho, tol=1e-11)
    assert st.rel_residual <= 1e-11
    p_gpu = ps.pressure64.cpu().numpy()
    rhs, ff = ps.rhs.cpu().numpy(), sim.fluid_fraction.cpu().numpy()
    # the operator's cell size as the solver passes it (float32, as the reference passes FIELD_DTYPE(dx))
    delta = float(np.float32(scene.dx))
    p_ref, hist = oracle.fp64_pressure_solve(rhs, ff, scene.grid_shape, delta, tol=1e-12, max_cycles=400)
    assert hist[-1] <= 1e-12
    fluid = np.zeros(scene.grid_shape, bool)
    fluid[1:-1, 1:-1, 1:-1] = ff[1:-1, 1:-1, 1:-1] > 0
    diff = np.linalg.norm((p_gpu - p_ref)[fluid]) / np.linalg.norm(p_ref[fluid])
    assert diff < 1e-8, diff
    assert backend.device_error() == 0
