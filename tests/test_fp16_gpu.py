"""FP16 storage of the coarse multigrid levels (tolerance mode; no counterpart in the reference).

The FP16 levels hold the same operator (exactly: its entries are small integers) and scaled p and b;
the W-cycle stays within FP16 rounding of the FP32 one and the refined solves converge as fast."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from continuum_liquid_b200 import multigrid, pressure_solve, scenes, solver

pytestmark = pytest.mark.gpu
F32 = np.float32


def liquid_system(shape, seed):
    """Fluid fraction of a liquid slab with scattered air cells and a random velocity field."""
    rng = np.random.default_rng(seed)
    ff = np.zeros(shape, F32)
    ff[1:-1, 1 : shape[1] // 2 + 2, 1:-1] = 1.0
    ff[rng.random(shape) < 0.05] = 0
    ff[[0, -1]] = 0
    ff[:, [0, -1]] = 0
    ff[:, :, [0, -1]] = 0
    vel = [torch.from_numpy(rng.standard_normal(shape).astype(F32)).cuda() for _ in range(3)]
    return torch.from_numpy(ff).cuda(), vel


@pytest.mark.parametrize("shape", [(66, 66, 66), (80, 70, 60)])
def test_fp16_levels_and_operators(backend, shape):
    dx = 1.0 / shape[0]
    ff, vel = liquid_system(shape, 3)
    rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
    h32 = multigrid.MultigridHierarchy(backend, shape, dx)
    h16 = multigrid.MultigridHierarchy(backend, shape, dx, fp16_max_size=64)
    assert h16.fp16_level >= 1 and all(max(s) <= 64 for s in h16.shapes[h16.fp16_level:])
    assert all(max(s) > 64 for s in h16.shapes[1 : h16.fp16_level])
    for h in (h32, h16):
        h.rhs_operator(vel, ff, rhs, 1.0 / 240.0, 1000.0)
        h.build_coarse()
    assert h16.fp16_inexact_entries() == 0
    for level in range(1, h16.levels):
        a, b = h32.level_arrays(level), h16.level_arrays(level)
        assert np.array_equal(a["mask"], b["mask"])
        assert np.array_equal(a["op"], b["op"])  # the FP16 operator is exact
        assert h16.op[level].dtype == (torch.float16 if h16.is_fp16(level) else torch.float32)
    # one W-cycle from zero on the same right-hand side: FP16 rounding only
    for h in (h32, h16):
        h.residual_norms(torch.zeros_like(rhs), rhs)  # norms[0] = ||rhs||^2 for the FP16 scales
    e32, e16 = torch.zeros_like(rhs), torch.zeros_like(rhs)
    h32.w_cycle(e32, rhs)
    h16.w_cycle(e16, rhs)
    scale = h16.fp16_scale.cpu().numpy()
    assert scale[0] > 0 and 0.5 <= scale[2] < 1.0
    rel = float(torch.linalg.norm(e16 - e32) / torch.linalg.norm(e32))
    assert rel < 5e-3, rel
    assert backend.device_error() == 0


@pytest.mark.parametrize("bottom", [1, 0])
def test_fp16_refined_solve_holds_convergence(backend, bottom):
    shape = (66, 66, 66)
    dx = 1.0 / 66
    ff, vel = liquid_system(shape, 7)
    backend.lib.clb_mg_set_option(0, bottom)
    try:
        cycles = {}
        for fp16 in (False, True):
            ps = pressure_solve.PressureSolver(backend, shape, dx, coarse_fp16=fp16, autotune=False)
            p = torch.zeros(shape, dtype=torch.float32, device="cuda")
            st = ps.solve(vel, ff, p, 1.0 / 240.0, 1000.0, tol=1e-6)
            assert st.rel_residual <= 1e-6
            assert ps.relative_residual(ps.pressure64) == pytest.approx(st.rel_residual, rel=1e-9)
            cycles[fp16] = st.cycles
        assert cycles[True] <= cycles[False] + 1, cycles
    finally:
        backend.lib.clb_mg_set_option(0, 1)
    assert backend.device_error() == 0


def test_fp16_parity_mode_is_refused(backend):
    ps = pressure_solve.PressureSolver(backend, (34, 34, 34), 1.0 / 34, coarse_fp16=True)
    assert ps.hierarchy.fp16_level > 0
    z = torch.zeros((34, 34, 34), dtype=torch.float32, device="cuda")
    with pytest.raises(ValueError, match="tolerance"):
        ps.solve((z, z, z), z, z.clone(), 1.0 / 240.0, 1000.0, tol=None)


def test_full_steps_with_fp16_coarse_levels(backend):
    s = scenes.block(48)
    pos, vel = scenes.seed_particles(s)
    totals = {}
    for fp16 in (False, True):
        opts = solver.StepOptions(flip_ratio=0.95, tol=1e-6, gravity=s.gravity, coarse_fp16=fp16)
        sim = solver.FlipSolver(backend, s.grid_shape, s.dx, pos, vel, dt=s.dt, options=opts)
        stats = [sim.step() for _ in range(5)]
        assert all(st.rel_residual <= 1e-6 for st in stats)
        totals[fp16] = sum(st.cycles for st in stats)
        if fp16:
            assert sim.pressure_solver.hierarchy.fp16_level > 0
    assert totals[True] <= totals[False] + 5, totals
    assert backend.device_error() == 0


@pytest.mark.parametrize("kind", [2, 3, 5, 6])
def test_fp16_fused_sweeps_equal_per_cell_sweeps(backend, kind):
    """The fused FP16 sweep kinds round every update to FP16 as the per-cell kind stores it: the same
    values on every FP16 level, for odd and even iteration counts."""
    shape = (80, 70, 60)
    dx = 1.0 / 80
    ff, vel = liquid_system(shape, 11)
    rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
    h = multigrid.MultigridHierarchy(backend, shape, dx, fp16_max_size=64, fused_min_cells=1)
    h.rhs_operator(vel, ff, rhs, 1.0 / 240.0, 1000.0)
    h.build_coarse()
    h.residual_norms(torch.zeros_like(rhs), rhs)
    e = torch.zeros_like(rhs)
    h.w_cycle(e, rhs)  # fills every level's p and b with scaled FP16 values
    levels = [l for l in range(1, h.levels - 1) if h.is_fp16(l)]
    assert levels
    for level in levels:
        start_p = h.p[level].clone()
        for iterations in (1, 2, 3):
            results = {}
            for k in (4, kind):
                h.set_sweep(level, k)
                h.p[level].copy_(start_p)
                h.smooth(level, iterations)
                results[k] = h.p[level].clone()
            assert torch.equal(results[4], results[kind]), (level, iterations)
            assert results[4].abs().max() > 0
    assert backend.device_error() == 0


@pytest.mark.parametrize("scale,cs", [(1.0, None), (1.7, None), (1.8, (1, 0))])
@pytest.mark.parametrize("shape", [(130, 130, 130), (134, 120, 125)])
def test_fp16_cluster_visit_equals_level_by_level(backend, shape, scale, cs):
    """With FP16 storage the cluster visit of the third-coarsest level (and its bottom visits) rounds
    exactly where the level-by-level kernels store FP16: W-cycles agree bit for bit."""
    dx = 1.0 / shape[0]
    ff, vel = liquid_system(shape, 13)
    rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
    h = multigrid.MultigridHierarchy(backend, shape, dx, fp16_max_size=64)
    assert h.fp16_level == h.levels - 3
    h.rhs_operator(vel, ff, rhs, 1.0 / 240.0, 1000.0)
    h.build_coarse()
    h.residual_norms(torch.zeros_like(rhs), rhs)
    out = {}
    try:
        for cluster in (0, 1):
            backend.lib.clb_mg_set_option(2, cluster)
            e = torch.zeros_like(rhs)
            for _ in range(2):
                h.w_cycle(e, rhs, prolong_scale=scale, coarse_smooth=cs)
            out[cluster] = e
    finally:
        backend.lib.clb_mg_set_option(2, 1)
    assert torch.equal(out[0], out[1])
    assert out[1].abs().max() > 0
    assert backend.device_error() == 0

