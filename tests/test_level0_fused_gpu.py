"""The fused level-0 visit of the W-cycle (sweep kind 7, csrc/mg_level0.cuh): pre-smoothing with the
residual and restriction in one launch, prolongation with post-smoothing in one, on 3-D fluid tiles.
Its values must be the launch-per-step W-cycle's, bit for bit, and so the oracle's."""

import numpy as np
import pytest
import torch

from continuum_liquid_b200 import multigrid, pressure_solve

pytestmark = pytest.mark.gpu

F32 = np.float32


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def corner_system(shape, seed):
    rng = np.random.default_rng(seed)
    ff = np.zeros(shape, F32)
    nx, ny, nz = shape
    ff[1 : (2 * nx) // 3, 1 : (7 * ny) // 10, 1 : nz // 2] = 1.0
    ff[rng.random(shape) < 0.03] = 0
    u, v, w = (rng.standard_normal(shape).astype(F32) for _ in range(3))
    return ff, u, v, w


def built_hierarchy(backend, shape, dx, ff, u, v, w, **kw):
    h = multigrid.MultigridHierarchy(backend, shape, float(dx), **kw)
    rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
    h.rhs_operator((dev(u), dev(v), dev(w)), dev(ff), rhs, 1.0 / 240.0, 1000.0)
    h.build_coarse()
    return h, rhs


@pytest.mark.parametrize("shape", [(66, 70, 68), (40, 36, 44), (64, 64, 64), (35, 26, 99)])
@pytest.mark.parametrize("smooth", [(1, 1), (2, 4), (1, 2), (3, 1)])
def test_fused_level0_w_cycle_matches_oracle(backend, oracle, shape, smooth):
    """Kind 7 from a stale correction (x_from_zero) gives the reference's W-cycle from zero."""
    pre, post = smooth
    dx = F32(1.0 / shape[0])
    ff, u, v, w = corner_system(shape, 61)
    h, rhs = built_hierarchy(backend, shape, dx, ff, u, v, w)
    assert int(h.fused_tile_count.item()) > 0
    assert int(h.fused_tile_count.item()) < int(backend.lib.clb_mg_fused_tile_capacity(*shape))
    P = torch.zeros(shape, dtype=torch.float32, device="cuda")
    h.w_cycle(P, rhs, pre_smooth=pre, post_smooth=post, coarse_iterations=8, x_zero_outside=True)
    assert P.abs().max() > 0  # a previous correction the next W-cycle must ignore
    h.set_sweep(0, 7)
    before = backend.launch_count()
    h.w_cycle(P, rhs, pre_smooth=pre, post_smooth=post, coarse_iterations=8, x_from_zero=True)
    fused_launches = backend.launch_count() - before
    orhs = oracle.pressure_rhs(u, v, w, ff, dx, 1.0 / 240.0, 1000.0, shape)
    oops = oracle.build_finest_operator(ff, shape)
    q = np.zeros(shape, F32)
    oracle.Levels(shape).w_cycle(q, orhs, ff, oops, dx, pre=pre, post=post, coarse=8)
    assert np.array_equal(host(P), q)
    # the launch-per-step path from the same stale correction: same values, 2 (pre + post) + 2 more launches
    h.set_sweep(0, 1)
    P2 = torch.zeros(shape, dtype=torch.float32, device="cuda")
    h.w_cycle(P2, rhs, pre_smooth=pre, post_smooth=post, coarse_iterations=8, x_zero_outside=True)
    before = backend.launch_count()
    h.w_cycle(P2, rhs, pre_smooth=pre, post_smooth=post, coarse_iterations=8, x_from_zero=True)
    plain_launches = backend.launch_count() - before
    assert np.array_equal(host(P2), q)
    assert plain_launches - fused_launches == (pre + post) + 2
    assert backend.device_error() == 0


def test_fused_level0_keeps_zero_outside_the_fluid(backend):
    """Cells without fluid stay 0 in x after fused W-cycles, even where the second buffer holds values
    from an earlier use (the invariant the FCG step relies on)."""
    shape = (48, 40, 72)
    dx = F32(1.0 / 48)
    ff, u, v, w = corner_system(shape, 62)
    h, rhs = built_hierarchy(backend, shape, dx, ff, u, v, w)
    h.alt[0].fill_(3.0)  # stale values everywhere in the second buffer
    h.set_sweep(0, 7)
    P = torch.zeros(shape, dtype=torch.float32, device="cuda")
    for _ in range(3):
        h.w_cycle(P, rhs, pre_smooth=1, post_smooth=1, coarse_iterations=4, x_from_zero=True)
    fluid = (host(h.op0) & 64) != 0
    got = host(P)
    assert (got[~fluid] == 0).all()
    assert np.abs(got[fluid]).max() > 0


@pytest.mark.parametrize("fp16", [False, True])
def test_fused_level0_solve_equals_unfused(backend, fp16):
    """Tolerance-mode solves with and without the fused level-0 visit (graphs, FCG, FP16 coarse levels
    of at most 64 cells per side): the same cycles, residuals and FP64 pressure, bit for bit."""
    shape = (130, 130, 130)
    dx = F32(1.0 / 130)
    ff, u, v, w = corner_system(shape, 63)
    results = []
    for fused in (True, False):
        ps = pressure_solve.PressureSolver(backend, shape, float(dx), coarse_fp16=fp16, coarse_iterations=4,
                                           pre_smooth=1, post_smooth=1, fused_level0=fused)
        P = torch.zeros(shape, dtype=torch.float32, device="cuda")
        stats = ps.solve((dev(u), dev(v), dev(w)), dev(ff), P, 1.0 / 240.0, 1000.0, tol=1e-6)
        assert stats.rel_residual <= 1e-6
        if fp16:
            assert ps.hierarchy.fp16_level == 2
        results.append((stats.cycles, stats.rel_residual, host(ps.pressure64), host(P)))
    assert results[0][0] == results[1][0]
    assert results[0][1] == results[1][1]
    assert np.array_equal(results[0][2], results[1][2])
    assert np.array_equal(results[0][3], results[1][3])
    assert backend.device_error() == 0
