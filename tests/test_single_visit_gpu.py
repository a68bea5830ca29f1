"""The W-cycle with levels visited once per parent visit from a given level on (clb_mg_set_option 4,
a preconditioner variant of the tolerance mode) against the oracle's restatement of the same
recursion, on every path: level by level, the bottom visit and the cluster visit."""

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


@pytest.fixture
def options(backend):
    yield backend
    for option, default in ((0, 1), (2, 1), (4, 0)):
        backend.call("clb_mg_set_option", option, default)


def system(shape, seed):
    rng = np.random.default_rng(seed)
    ff = np.zeros(shape, F32)
    nx, ny, nz = shape
    ff[1 : (2 * nx) // 3, 1 : (3 * ny) // 4, 1 : nz - 1] = 1.0
    ff[rng.random(shape) < 0.03] = 0
    u, v, w = (rng.standard_normal(shape).astype(F32) for _ in range(3))
    return ff, u, v, w


@pytest.mark.parametrize("shape", [(130, 130, 130), (66, 70, 68), (40, 36, 44)])
@pytest.mark.parametrize("single", [1, 2, 3])
@pytest.mark.parametrize("paths", ["all", "level_by_level"])
def test_single_visit_w_cycle_matches_oracle(options, oracle, shape, single, paths):
    backend = options
    dx = F32(1.0 / shape[0])
    ff, u, v, w = system(shape, 81)
    h = multigrid.MultigridHierarchy(backend, shape, float(dx))
    if single >= h.levels:
        pytest.skip("no such level")
    rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
    h.rhs_operator((dev(u), dev(v), dev(w)), dev(ff), rhs, 1.0 / 240.0, 1000.0)
    h.build_coarse()
    backend.call("clb_mg_set_option", 4, single)
    if paths == "level_by_level":
        backend.call("clb_mg_set_option", 0, 0)
        backend.call("clb_mg_set_option", 2, 0)
    P = torch.zeros(shape, dtype=torch.float32, device="cuda")
    for _ in range(2):
        h.w_cycle(P, rhs, pre_smooth=1, post_smooth=2, coarse_iterations=6, x_zero_outside=True)
    orhs = oracle.pressure_rhs(u, v, w, ff, dx, 1.0 / 240.0, 1000.0, shape)
    oops = oracle.build_finest_operator(ff, shape)
    q = np.zeros(shape, F32)
    levels = oracle.Levels(shape)
    for _ in range(2):
        levels.w_cycle(q, orhs, ff, oops, dx, pre=1, post=2, coarse=6, single_from=single)
    assert np.array_equal(host(P), q)
    # and it is a different preconditioner from the reference's W-cycle
    q2 = np.zeros(shape, F32)
    oracle.Levels(shape).w_cycle(q2, orhs, ff, oops, dx, pre=1, post=2, coarse=6)
    assert not np.array_equal(q, q2)
    assert backend.device_error() == 0


def test_single_visit_fcg_history_matches_oracle(options, oracle):
    backend = options
    shape, dx = (66, 60, 70), F32(1.0 / 66)
    ff, u, v, w = system(shape, 82)
    backend.call("clb_mg_set_option", 4, 2)
    ps = pressure_solve.PressureSolver(backend, shape, float(dx), autotune=False, coarse_iterations=4, pre_smooth=1,
                                       post_smooth=1)
    P = torch.zeros(shape, dtype=torch.float32, device="cuda")
    dt, rho = 1.0 / 240.0, 1000.0
    ps.solve((dev(u), dev(v), dev(w)), dev(ff), P, dt, rho, tol=1e-3, use_graph=False)
    h = ps.hierarchy
    rng = np.random.default_rng(9)
    p0 = rng.standard_normal(shape).astype(F32) * 10.0
    ps.cur = 0
    backend.call("clb_mg_ir_init", dev(p0), h.op0, ps.p64[0], *shape)
    got = [ps._relative(h.residual_norms(ps.p64[0], ps.rhs, r_out=ps.residual))]
    ps.direction[0].zero_()
    ps.fcg_state.zero_()
    for _ in range(8):
        ps._refine(use_graph=False)
        got.append(ps._relative(h.norms))
    orhs = oracle.pressure_rhs(u, v, w, ff, dx, dt, rho, shape)
    x, want = oracle.fcg_solve(orhs, ff, shape, dx, p0=p0, tol=0.0, max_cycles=8, coarse_iterations=4, pre_smooth=1,
                               post_smooth=1, single_from=2)
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-14)  # FP64 summation orders differ
    assert want[-1] < 1e-3 * want[0]
    np.testing.assert_allclose(host(ps.pressure64), x, rtol=0, atol=1e-9 * np.abs(x).max())
