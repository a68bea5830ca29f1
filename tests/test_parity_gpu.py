"""GPU parity: every CUDA entry point against the oracle on the same seeded inputs.

Equality here is IEEE value equality (numpy.array_equal: -0 == +0). Everything except the
documented tolerance cases must match exactly; the whole library is compiled without FMA
contraction and keeps the reference's evaluation orders.
"""

import numpy as np
import pytest
import torch

from continuum_liquid_b200 import boundary_conditions, multigrid, particles, pressure_solve, scenes, solver
from continuum_liquid_b200 import velocity_update, voxelise_mesh

pytestmark = pytest.mark.gpu

F32 = np.float32


def dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def scene_particles(n, seed=0, jitter_vel=True, shape=None):
    s = scenes.dam_break(n, seed)
    if shape is not None:
        s.grid_shape = shape
    pos, vel = scenes.seed_particles(s)
    if jitter_vel:
        vel = np.random.default_rng(seed + 1).standard_normal(pos.shape).astype(F32)
    return s, pos, vel


@pytest.fixture(params=[(16, 16, 16), (33, 33, 33), (40, 24, 31), (24, 20, 32)], ids=lambda s: "x".join(map(str, s)))
def case(request):
    shape = request.param
    n = shape[0]
    s, pos, vel = scene_particles(n, seed=n, shape=shape)
    s.grid_shape = shape
    s.dx = 1.0 / n
    pos = pos[np.all(pos < np.asarray(shape, F32) * F32(s.dx), axis=1)]
    vel = vel[: len(pos)]
    return shape, F32(s.dx), pos, vel


# ---- binning, scan, sort, P2G ---------------------------------------------------------------------
def test_count_keys_ranks(backend, oracle, case):
    shape, dx, pos, _ = case
    C, n = int(np.prod(shape)), len(pos)
    counts = torch.zeros(C, dtype=torch.int32, device="cuda")
    keys = torch.zeros(n, dtype=torch.int32, device="cuda")
    ranks = torch.zeros(n, dtype=torch.int32, device="cuda")
    particles.count_particles_per_cell(backend, None, dev(pos), counts, n, shape, dx, keys, ranks)
    assert np.array_equal(host(counts), oracle.count_particles(pos, dx, shape))
    k = host(keys)
    assert np.array_equal(k, oracle.bin_keys(pos, dx, shape))
    r = host(ranks)
    order = np.lexsort((r, k))
    # ranks within each bin are exactly 0..count-1
    kk, rr = k[order], r[order]
    starts = np.r_[0, np.flatnonzero(np.diff(kk)) + 1]
    expect = np.arange(n) - np.repeat(starts, np.diff(np.r_[starts, n]))
    assert np.array_equal(rr, expect)


@pytest.mark.parametrize("size", [0, 1, 5, 4095, 4096, 4097, 100003, 16777216 + 77])
def test_scan(backend, size):
    rng = np.random.default_rng(size)
    values = rng.integers(0, 9, size).astype(np.int32)
    out = torch.zeros(max(size, 1), dtype=torch.int32, device="cuda")[:size]
    total = torch.zeros(1, dtype=torch.int32, device="cuda")
    scratch = torch.zeros(backend.scan_scratch_bytes(size), dtype=torch.uint8, device="cuda")
    backend.call("clb_exclusive_prefix_sum", dev(values) if size else out, out, total, size, scratch,
                 scratch.numel())
    expect = (np.cumsum(values) - values).astype(np.int64)
    assert np.array_equal(host(out).astype(np.int64), expect)
    assert int(host(total)[0]) == int(values.sum())
    assert backend.device_error() == 0


def test_scan_rejects_small_scratch(backend):
    values = torch.ones(10000, dtype=torch.int32, device="cuda")
    scratch = torch.zeros(8, dtype=torch.uint8, device="cuda")
    with pytest.raises(RuntimeError, match="scratch"):
        backend.call("clb_exclusive_prefix_sum", values, values, None, 10000, scratch, 8)


def test_particle_to_grid_stage_bit_exact(backend, oracle, case):
    shape, dx, pos, vel = case
    n = len(pos)
    work, vwork, counts, outs, sums = particles.create_particle_sort_buffers(backend, shape, n)
    grid = [torch.zeros(shape, dtype=torch.float32, device="cuda") for _ in range(4)]
    P, V = dev(pos), dev(vel)
    res = particles.particle_to_grid(backend, None, P, V, work, vwork, tuple(grid[:3]), counts, outs, sums, grid[3],
                                     n, shape, float(dx), 8)
    pos_s, vel_s, u, v, w, ff, ocounts, ooffsets = oracle.particle_to_grid(pos, vel, dx, shape)
    assert res[0] is work and res[2] is P  # buffers swapped like particles.py:188-192
    assert np.array_equal(host(counts), ocounts)
    assert np.array_equal(host(outs[0]), ooffsets)
    assert np.array_equal(host(res[0]), pos_s)
    assert np.array_equal(host(res[1]), vel_s)
    for g, o in zip(grid, (u, v, w, ff)):
        assert np.array_equal(host(g), o)


@pytest.mark.parametrize("shape", [(12, 12, 12), (12, 12, 32)])
def test_dense_bins_and_outside_particles(backend, oracle, shape):
    """Many particles in one bin (slow path of the stable sort), in grids whose rows are and are not a
    multiple of the 32-cell gather block, and particles outside the grid (clamped bins), as the
    reference allows."""
    dx = F32(1.0 / 12)
    rng = np.random.default_rng(5)
    dense = (np.array([5.6, 5.6, 5.6]) + rng.random((300, 3)) * 0.3) * dx
    outside = np.array([[-0.2, 0.5, 0.5], [0.5, 1.7, 0.5], [0.5, 0.5, -3.0]])
    pos = np.concatenate([dense, rng.random((200, 3)), outside]).astype(F32)
    vel = rng.standard_normal(pos.shape).astype(F32)
    n = len(pos)
    work, vwork, counts, outs, sums = particles.create_particle_sort_buffers(backend, shape, n)
    grid = [torch.zeros(shape, dtype=torch.float32, device="cuda") for _ in range(4)]
    res = particles.particle_to_grid(backend, None, dev(pos), dev(vel), work, vwork, tuple(grid[:3]), counts, outs,
                                     sums, grid[3], n, shape, float(dx), 8)
    pos_s, vel_s, u, v, w, ff, _, _ = oracle.particle_to_grid(pos, vel, dx, shape)
    assert np.array_equal(host(res[0]), pos_s) and np.array_equal(host(res[1]), vel_s)
    for g, o in zip(grid, (u, v, w, ff)):
        assert np.array_equal(host(g), o)


def test_empty_particle_set(backend):
    shape = (8, 8, 8)
    work, vwork, counts, outs, sums = particles.create_particle_sort_buffers(backend, shape, 0)
    grid = [torch.ones(shape, dtype=torch.float32, device="cuda") for _ in range(4)]
    e = torch.zeros((1, 3), dtype=torch.float32, device="cuda")
    particles.particle_to_grid(backend, None, e, e.clone(), work, vwork, tuple(grid[:3]), counts, outs, sums,
                               grid[3], 0, shape, 0.125, 8)
    assert not any(host(g).any() for g in grid)


# ---- G2P and the fused particle update -----------------------------------------------------------
@pytest.mark.parametrize("flip_ratio", [1.0, 0.95])
def test_grid_to_particle(backend, oracle, case, flip_ratio):
    shape, dx, pos, vel = case
    rng = np.random.default_rng(7)
    cur = [rng.standard_normal(shape).astype(F32) for _ in range(3)]
    old = [rng.standard_normal(shape).astype(F32) for _ in range(3)]
    V = dev(vel)
    particles.grid_to_particle(backend, None, V, dev(pos), tuple(dev(a) for a in cur), tuple(dev(a) for a in old),
                               len(pos), shape, float(dx), flip_ratio)
    assert np.array_equal(host(V), oracle.grid_to_particle(vel, pos, cur, old, dx, shape, flip_ratio))


@pytest.mark.parametrize("with_obstacle", [False, True])
def test_fused_particle_update(backend, oracle, case, with_obstacle):
    shape, dx, pos, vel = case
    rng = np.random.default_rng(8)
    cur = [rng.standard_normal(shape).astype(F32) for _ in range(3)]
    old = [rng.standard_normal(shape).astype(F32) for _ in range(3)]
    dt = 1.0 / 60.0
    obstacle = (rng.random(shape) < 0.2).astype(np.uint8) if with_obstacle else np.zeros(shape, np.uint8)
    P, V, prev = dev(pos), dev(vel), torch.zeros(pos.shape, dtype=torch.float32, device="cuda")
    particles.particle_update(backend, None, P, V, tuple(dev(a) for a in cur), tuple(dev(a) for a in old),
                              dev(obstacle) if with_obstacle else None, len(pos), shape, float(dx), dt, 0.95,
                              previous_particles=prev)
    v2 = oracle.grid_to_particle(vel, pos, cur, old, dx, shape, 0.95)
    p2 = oracle.advect(pos, v2, dt)
    p2, v2 = oracle.particle_domain_bc(p2, v2, dx, shape)
    p2, v2 = oracle.particle_obstacle_bc(p2, pos, v2, obstacle, dx, shape)
    assert np.array_equal(host(prev), pos)
    assert np.array_equal(host(P), p2)
    assert np.array_equal(host(V), v2)


def test_separate_particle_kernels(backend, oracle, case):
    shape, dx, pos, vel = case
    rng = np.random.default_rng(9)
    obstacle = (rng.random(shape) < 0.2).astype(np.uint8)
    prev = (pos - rng.random(pos.shape).astype(F32) * F32(dx)).astype(F32)
    P, V = dev(pos), dev(vel)
    particles.advect_particles(backend, None, P, V, len(pos), 0.01)
    boundary_conditions.particle_domain_bc(backend, None, P, V, len(pos), shape, float(dx))
    boundary_conditions.particle_obstacle_bc(backend, None, P, dev(prev), V, dev(obstacle), len(pos), shape,
                                             float(dx))
    p2 = oracle.advect(pos, vel, 0.01)
    p2, v2 = oracle.particle_domain_bc(p2, vel, dx, shape)
    p2, v2 = oracle.particle_obstacle_bc(p2, prev, v2, obstacle, dx, shape)
    assert np.array_equal(host(P), p2) and np.array_equal(host(V), v2)


# ---- grid kernels ---------------------------------------------------------------------------------
def test_grid_kernels(backend, oracle, case):
    shape, dx, _, _ = case
    rng = np.random.default_rng(11)
    u, v, w = (rng.standard_normal(shape).astype(F32) for _ in range(3))
    ff = (rng.random(shape) * (rng.random(shape) < 0.6)).astype(F32)
    ff[[0, -1]] = 0
    ff[:, [0, -1]] = 0
    ff[:, :, [0, -1]] = 0
    obstacle = (rng.random(shape) < 0.1).astype(np.uint8)
    p = rng.standard_normal(shape).astype(F32)
    dt, rho, nu = 1.0 / 240.0, 1000.0, 1e-3
    # update_velocity
    out = [torch.zeros(shape, dtype=torch.float32, device="cuda") for _ in range(3)]
    velocity_update.update_velocity(backend, None, (dev(u), dev(v), dev(w)), tuple(out), dev(ff), (0.0, -9.81, 0.0),
                                    0.0, 0.0, 0.0, rho, nu, float(dx), dt, shape)
    exp = oracle.update_velocity(u, v, w, ff, (0.0, -9.81, 0.0), (0.0, 0.0, 0.0), rho, nu, dx, dt, shape)
    for a, b in zip(out, exp):
        assert np.array_equal(host(a), b)
    # grid_domain_bc
    U, Vv, W = dev(u), dev(v), dev(w)
    boundary_conditions.grid_domain_bc(backend, None, (U, Vv, W), shape)
    for a, b in zip((U, Vv, W), oracle.grid_domain_bc(u, v, w, shape)):
        assert np.array_equal(host(a), b)
    # grid_obstacle_bc (+ extrapolation)
    U, Vv, W, FF = dev(u), dev(v), dev(w), dev(ff)
    boundary_conditions.grid_obstacle_bc(backend, None, (U, Vv, W), FF, dev(obstacle), shape)
    for a, b in zip((U, Vv, W, FF), oracle.grid_obstacle_bc(u, v, w, ff, obstacle, shape)):
        assert np.array_equal(host(a), b)
    # pressure_rhs / pressure_correction / neumann
    rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
    backend.call("clb_pressure_rhs", dev(u), dev(v), dev(w), dev(ff), rhs, float(F32(rho / dt)), float(F32(1.0 / float(dx))),
                 *shape)
    assert np.array_equal(host(rhs), oracle.pressure_rhs(u, v, w, ff, dx, dt, rho, shape))
    U, Vv, W = dev(u), dev(v), dev(w)
    pressure_solve.pressure_correction(backend, None, (U, Vv, W), dev(p), float(dx), dt, rho, shape)
    for a, b in zip((U, Vv, W), oracle.pressure_correction(u, v, w, p, dx, dt, rho, shape)):
        assert np.array_equal(host(a), b)
    Pp = dev(p)
    boundary_conditions.neumann_domain_bc(backend, None, Pp, shape)
    assert np.array_equal(host(Pp), oracle.neumann_domain_bc(p, shape))


# ---- multigrid ------------------------------------------------------------------------------------
def random_system(shape, seed):
    rng = np.random.default_rng(seed)
    ff = np.zeros(shape, F32)
    ff[1:-1, 1 : shape[1] // 2 + 2, 1:-1] = 0.5
    ff[rng.random(shape) < 0.1] = 0
    ff[[0, -1]] = 0
    ff[:, [0, -1]] = 0
    ff[:, :, [0, -1]] = 0
    b = (rng.standard_normal(shape) * 1e4 * (ff > 0)).astype(F32)
    p0 = rng.standard_normal(shape).astype(F32)
    return ff, b, p0


def test_reference_layout_stage_functions(backend, oracle, case):
    """multigrid.smooth / coarse_smooth on the reference's level arrays (packed for the product kernels)
    equal the oracle's rbgs_step and coarse_smooth; the finest operator survives the byte packing."""
    shape, dx, _, _ = case
    ff, b, p0 = random_system(shape, 12)
    oops = oracle.build_finest_operator(ff, shape)
    op0 = torch.zeros(shape, dtype=torch.uint8, device="cuda")
    invalid = torch.zeros(1, dtype=torch.int32, device="cuda")
    backend.call("clb_mg_pack_finest", dev(ff), *(dev(o) for o in oops), op0, invalid, *shape)
    back = [torch.zeros(shape, dtype=torch.float32, device="cuda") for _ in range(4)]
    backend.call("clb_mg_unpack_finest", op0, *back, *shape)
    assert int(invalid.item()) == 0
    for a, o in zip(back, oops):
        assert np.array_equal(host(a), o)
    ops = tuple(dev(o) for o in oops)
    P = dev(p0)
    multigrid.smooth(backend, None, P, dev(b), dev(ff), ops, float(dx), 2, shape)
    q = p0.copy()
    for parity in (0, 1, 0, 1):
        oracle.lib().orc_rbgs_step_f32(q, b, ff, *oops, dx, parity, *shape)
    assert np.array_equal(host(P), q)
    # a coarse level as the reference's restriction makes it, then its coarse smooth
    cshape = tuple(oracle.coarse_grid_size(s) for s in shape)
    oc = [np.zeros(cshape, F32) for _ in range(7)]
    oracle.lib().orc_restrict_residual_f32(q, b, ff, *oops, *oc, dx, *shape, *cshape)
    cp = dev(np.random.default_rng(13).standard_normal(cshape).astype(F32) * (oc[2] > 0))
    ocp = host(cp).copy()
    multigrid.coarse_smooth(backend, None, cp, dev(oc[1]), dev(oc[2]), tuple(dev(o) for o in oc[3:]), float(dx), 66,
                            cshape)
    oracle.lib().orc_coarse_smooth_f32(ocp, oc[1], oc[2], *oc[3:], dx, 66, *cshape)
    assert np.array_equal(host(cp), ocp)


def test_reference_layout_w_cycle(backend, oracle):
    shape, dx = (34, 34, 34), F32(1.0 / 34)
    ff, b, p0 = random_system(shape, 14)
    lv = multigrid.create_multigrid_levels(backend, shape)
    ops = tuple(dev(o) for o in oracle.build_finest_operator(ff, shape))
    P = dev(p0)
    for _ in range(2):
        multigrid.w_cycle(backend, None, 0, lv[0], lv[1], lv[2], lv[3], P, dev(b), dev(ff), ops, float(dx),
                          lv[4], shape, 2, 4, 64)
    levels = oracle.Levels(shape)
    q = p0.copy()
    oops = oracle.build_finest_operator(ff, shape)
    for _ in range(2):
        levels.w_cycle(q, b, ff, oops, dx)
    assert np.array_equal(host(P), q)
    # the coarse operators and masks, where the reference's restriction leaves them
    for l in range(1, len(levels.shapes)):
        assert np.array_equal(host(lv[2][l - 1]), levels.m[l]), f"mask {l}"
        for a, o in zip(lv[3][l - 1], levels.ops[l]):
            assert np.array_equal(host(a), o), f"operator {l}"
    with pytest.raises(ValueError, match="level 0"):
        multigrid.w_cycle(backend, None, 1, lv[0], lv[1], lv[2], lv[3], P, dev(b), dev(ff), ops, float(dx), lv[4],
                          shape, 2, 4, 64)
    bad = (dev(oops[0] * 0.5), *ops[1:])
    with pytest.raises(ValueError, match="finest-level operator"):
        multigrid.w_cycle(backend, None, 0, lv[0], lv[1], lv[2], lv[3], P, dev(b), dev(ff), bad, float(dx), lv[4],
                          shape, 2, 4, 64)


def test_reference_layout_pressure_solve(backend, oracle):
    """pressure_solve.pressure_solve (the stage the add-on calls, on the reference's arrays) equals the
    oracle's pressure_solve: pressure, right-hand side and finest operator."""
    from continuum_liquid_b200 import pressure_solve as ps_mod

    shape, dx, dt, rho = (34, 30, 38), 1.0 / 34, 1.0 / 240, 1000.0
    rng = np.random.default_rng(21)
    u, v, w = (rng.standard_normal(shape).astype(F32) for _ in range(3))
    ff, _, p0 = random_system(shape, 22)
    lv = multigrid.create_multigrid_levels(backend, shape)
    rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
    op0 = tuple(torch.zeros(shape, dtype=torch.float32, device="cuda") for _ in range(4))
    P = dev(p0)
    ps_mod.pressure_solve(backend, backend, backend, None, (dev(u), dev(v), dev(w)), dev(ff), P, rhs, lv[0], lv[1],
                          lv[2], op0, lv[3], lv[4], dx, dt, rho, 2, shape)
    p_ref, rhs_ref, op_ref = oracle.pressure_solve(u, v, w, ff, p0, dx, dt, rho, 2, shape)
    assert np.array_equal(host(P), p_ref)
    assert np.array_equal(host(rhs), rhs_ref)
    for a, o in zip(op0, op_ref):
        assert np.array_equal(host(a), o)


@pytest.mark.parametrize("shape", [(34, 34, 34), (66, 66, 66), (48, 40, 56)])
def test_packed_w_cycle_equals_reference(backend, oracle, shape):
    dx = F32(1.0 / shape[0])
    rng = np.random.default_rng(15)
    u, v, w = (rng.standard_normal(shape).astype(F32) for _ in range(3))
    ff, _, p0 = random_system(shape, 16)
    dt, rho = 1.0 / 240.0, 1000.0
    h = multigrid.MultigridHierarchy(backend, shape, float(dx))
    rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
    h.rhs_operator((dev(u), dev(v), dev(w)), dev(ff), rhs, dt, rho)
    orhs = oracle.pressure_rhs(u, v, w, ff, dx, dt, rho, shape)
    oops = oracle.build_finest_operator(ff, shape)
    assert np.array_equal(host(rhs), orhs)
    unpacked = multigrid.unpack_op0(host(h.op0))
    inner = np.zeros(shape, bool)
    inner[1:-1, 1:-1, 1:-1] = True
    assert np.array_equal(unpacked[0], ((ff > 0) & inner).astype(F32))
    for a, o in zip(unpacked[1:], oops):
        assert np.array_equal(a, o)
    h.build_coarse()
    P = dev(p0)
    for _ in range(2):
        h.w_cycle(P, rhs)
    levels = oracle.Levels(shape)
    q = p0.copy()
    for _ in range(2):
        levels.w_cycle(q, orhs, ff, oops, dx)
    assert np.array_equal(host(P), q)
    # coarse operators equal the oracle's (its levels hold the last restriction's operator)
    for lvl in range(1, h.levels):
        arr = h.level_arrays(lvl)
        assert np.array_equal(arr["op"][..., 0], levels.ops[lvl][0])
        assert np.array_equal(arr["op"][..., 1], levels.ops[lvl][1])
        assert np.array_equal(arr["mask"].astype(F32), levels.m[lvl])
    # FP64 residual norms
    norms = host(h.residual_norms(P, rhs))
    f64 = lambda a: np.asarray(a, np.float64)  # noqa: E731 - the GPU evaluates the residual in FP64
    rr, bb = oracle.residual_norms(f64(q), f64(orhs), f64(ff), [f64(a) for a in oops], float(dx))
    assert norms[0] == pytest.approx(rr, rel=1e-12) and norms[1] == pytest.approx(bb, rel=1e-12)


@pytest.mark.parametrize("method", ["fcg", "refine"])
def test_iterative_refinement_reaches_tolerance(backend, oracle, method):
    shape, dx = (34, 34, 34), F32(1.0 / 34)
    rng = np.random.default_rng(17)
    u, v, w = (rng.standard_normal(shape).astype(F32) for _ in range(3))
    ff, _, _ = random_system(shape, 18)
    dt, rho = 1.0 / 240.0, 1000.0
    ps = pressure_solve.PressureSolver(backend, shape, float(dx), method=method)
    P = torch.zeros(shape, dtype=torch.float32, device="cuda")
    stats = ps.solve((dev(u), dev(v), dev(w)), dev(ff), P, dt, rho, tol=1e-6)
    assert stats.rel_residual <= 1e-6
    assert stats.cycles >= 3
    orhs = oracle.pressure_rhs(u, v, w, ff, dx, dt, rho, shape)
    p64, hist = oracle.fp64_pressure_solve(orhs, ff, shape, dx, tol=1e-13)
    got = host(P)
    interior = ff > 0
    err = np.abs(got[interior] - p64[interior]).max() / np.abs(p64[interior]).max()
    assert err < 1e-5
    # the FP64 pressure is the solution: its own residual is the reported one
    assert ps.solved64
    got64 = host(ps.pressure64)
    err64 = np.abs(got64[interior] - p64[interior]).max() / np.abs(p64[interior]).max()
    assert err64 < 1e-5
    assert ps.relative_residual(ps.pressure64) == pytest.approx(stats.rel_residual, rel=1e-9)
    # air cells inside the domain hold zero pressure; ghosts carry the Neumann copy
    inner = np.zeros(shape, bool)
    inner[1:-1, 1:-1, 1:-1] = True
    assert not got[inner & (ff <= 0)].any()
    assert np.array_equal(got, oracle.neumann_domain_bc(got, shape))


@pytest.mark.parametrize("method,coarse,smooth,w,cs", [("fcg", 64, (2, 4), 1.0, None), ("refine", 64, (2, 4), 1.0, None),
                                                       ("fcg", 4, (2, 4), 1.0, None), ("fcg", 0, (2, 4), 1.0, None),
                                                       ("fcg", 4, (1, 1), 1.0, None), ("fcg", 4, (1, 2), 1.0, None),
                                                       ("fcg", 4, (1, 1), 1.7, None), ("refine", 4, (1, 1), 1.7, None),
                                                       ("fcg", 0, (1, 1), 1.8, (1, 0)), ("fcg", 0, (1, 2), 1.8, (1, 0))])
def test_refinement_history_matches_oracle(backend, oracle, method, coarse, smooth, w, cs):
    """Every W-cycle of the GPU iteration against the oracle's restatement (same FP32 W-cycle, with
    the reference's or fewer coarsest-level iterations, FP64 accumulation and scalars; only summation
    orders differ)."""
    shape, dx = (34, 30, 38), F32(1.0 / 34)
    rng = np.random.default_rng(5)
    u, v, w_vel = (rng.standard_normal(shape).astype(F32) for _ in range(3))
    ff, _, _ = random_system(shape, 6)
    dt, rho = 1.0 / 240.0, 1000.0
    ps = pressure_solve.PressureSolver(backend, shape, float(dx), method=method, autotune=False,
                                       coarse_iterations=coarse, pre_smooth=smooth[0], post_smooth=smooth[1],
                                       prolong_scale=w, coarse_smooth=cs)
    P = torch.zeros(shape, dtype=torch.float32, device="cuda")
    ps.solve((dev(u), dev(v), dev(w_vel)), dev(ff), P, dt, rho, tol=1e-3, use_graph=False)  # builds the system
    h = ps.hierarchy
    p0 = rng.standard_normal(shape).astype(F32) * 10.0
    ps.cur = 0
    backend.call("clb_mg_ir_init", dev(p0), h.op0, ps.p64[0], *shape)
    got = [ps._relative(h.residual_norms(ps.p64[0], ps.rhs, r_out=ps.residual))]
    ps.direction[0].zero_()
    ps.fcg_state.zero_()
    for _ in range(8):
        ps._refine(use_graph=False)
        got.append(ps._relative(h.norms))
    orhs = oracle.pressure_rhs(u, v, w_vel, ff, dx, dt, rho, shape)
    x, want = oracle.fcg_solve(orhs, ff, shape, dx, p0=p0, tol=0.0, max_cycles=8, flexible=(method == "fcg"),
                               coarse_iterations=coarse, pre_smooth=smooth[0], post_smooth=smooth[1],
                               prolong_scale=w, coarse_smooth=cs)
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-14)  # FP64 summation orders differ
    assert want[-1] < 1e-3 * want[0]
    scale = np.abs(x).max()
    np.testing.assert_allclose(host(ps.pressure64), x, rtol=0, atol=1e-9 * scale)


def test_fcg_needs_fewer_cycles_than_refinement(backend):
    s = scenes.block(48)
    counts = {}
    for method in ("refine", "fcg"):
        opts = solver.StepOptions(flip_ratio=0.95, tol=1e-6, gravity=s.gravity, method=method)
        pos, vel = scenes.seed_particles(s)
        sim = solver.FlipSolver(backend, s.grid_shape, s.dx, pos, vel, dt=s.dt, options=opts)
        stats = [sim.step() for _ in range(6)]
        assert all(st.rel_residual <= 1e-6 for st in stats)
        counts[method] = sum(st.cycles for st in stats)
    assert counts["fcg"] < counts["refine"], counts


def test_fp64_projection_matches_numpy(backend):
    shape = (20, 18, 22)
    rng = np.random.default_rng(3)
    u, v, w = (rng.standard_normal(shape).astype(F32) for _ in range(3))
    p = rng.standard_normal(shape) * 1e3
    dtr, inv_dx = F32(1.0 / 240.0 / 1000.0), F32(20.0)
    U, V, W = dev(u), dev(v), dev(w)
    P = torch.from_numpy(p).cuda()
    backend.call("clb_neumann_domain_bc_f64", P, *shape)
    backend.call("clb_pressure_correction_f64", U, V, W, P, float(dtr), float(inv_dx), *shape)
    q = p.copy()
    nx, ny, nz = shape
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                if not (0 < i < nx - 1 and 0 < j < ny - 1 and 0 < k < nz - 1):
                    q[i, j, k] = p[min(max(i, 1), nx - 2), min(max(j, 1), ny - 2), min(max(k, 1), nz - 2)]
    assert np.array_equal(host(P), q)
    I = (slice(1, -1),) * 3
    want = [a.copy() for a in (u, v, w)]
    grads = (q[2:, 1:-1, 1:-1], q[1:-1, 2:, 1:-1], q[1:-1, 1:-1, 2:])
    for a, nb in zip(want, grads):
        g = (nb - q[I]) * np.float64(inv_dx)
        a[I] = (a[I].astype(np.float64) - np.float64(dtr) * g).astype(F32)
    for got, a in zip((U, V, W), want):
        assert np.array_equal(host(got), a)


# ---- voxelisation ---------------------------------------------------------------------------------
@pytest.mark.parametrize("n,sub", [(32, 2), (48, 3), (40, 4)])
def test_voxelise_bit_exact(backend, oracle, n, sub):
    shape, delta = (n, n, n), 1.0 / n
    origin = (-0.5, -0.5, 0.0)
    rng = np.random.default_rng(n)
    tris = scenes.icosphere(sub, 0.21, (rng.uniform(-0.1, 0.1), rng.uniform(-0.1, 0.1), 0.5))
    expect = oracle.voxelise(tris, shape, delta, origin)
    for cull in (False, True):
        mask = torch.zeros(shape, dtype=torch.uint8, device="cuda")
        voxelise_mesh.voxelise_triangles(backend, None, tris, mask, shape, delta, origin, cull=cull)
        assert np.array_equal(host(mask), expect), f"cull={cull}"
    assert expect.sum() > 0


def test_voxelise_direction_matches_oracle(backend, oracle):
    assert np.array_equal(np.asarray(backend.voxelise_direction, F32), oracle.voxelise_direction())


# ---- whole steps -----------------------------------------------------------------------------------
@pytest.mark.parametrize("with_obstacle", [False, True])
def test_full_steps_match_oracle(backend, oracle, with_obstacle):
    n = 32
    s = scenes.collider_pool(n, subdivisions=2) if with_obstacle else scenes.dam_break(n)
    obstacle = np.zeros(s.grid_shape, np.uint8)
    for tris in s.obstacles:
        obstacle = oracle.voxelise(tris, s.grid_shape, s.dx, s.origin, obstacle)
    pos, vel = scenes.seed_particles(s, obstacle)
    opts = solver.StepOptions(flip_ratio=1.0, num_vcycles=1, gravity=s.gravity, use_graph=False)
    sim = solver.FlipSolver(backend, s.grid_shape, s.dx, pos, vel, obstacle=obstacle, dt=s.dt, options=opts)
    ref = oracle.OracleSim(s.grid_shape, s.dx, pos, vel, obstacle=obstacle, dt=s.dt, flip_ratio=1.0,
                           gravity=s.gravity)
    for step in range(4):
        sim.step()
        ref.step()
        assert np.array_equal(host(sim.pressure), ref.pressure), f"pressure, step {step}"
        assert np.array_equal(sim.positions(), ref.pos), f"positions, step {step}"
        assert np.array_equal(sim.velocities(), ref.vel), f"velocities, step {step}"


def test_bad_arguments_raise(backend):
    t = torch.zeros(8, dtype=torch.float32, device="cuda")
    with pytest.raises(RuntimeError, match="grid"):
        backend.call("clb_grid_domain_bc", t, t, t, 2, 2, 2)
    with pytest.raises(RuntimeError, match="negative iterations"):
        backend.call("clb_mg_smooth_level", t, t, t, t, 1.0, -1, 4, 4, 4)


@pytest.mark.parametrize("cluster", [1, 0])
@pytest.mark.parametrize("pdl", [1, 0])
@pytest.mark.parametrize("bottom", [1, 0])
@pytest.mark.parametrize("shape", [(66, 66, 66), (34, 40, 30), (70, 66, 61)])
def test_w_cycle_paths_agree(backend, oracle, shape, bottom, pdl, cluster):
    """The cluster visit, the single-block bottom visit and the fused red-black iterations give the
    reference values, with and without programmatic dependent launch."""
    dx = F32(1.0 / shape[0])
    ff, b, p0 = random_system(shape, 21)
    backend.lib.clb_mg_set_option(0, bottom)
    backend.lib.clb_mg_set_option(1, pdl)
    backend.lib.clb_mg_set_option(2, cluster)
    try:
        h = multigrid.MultigridHierarchy(backend, shape, float(dx))
        h.op0.copy_(torch.zeros_like(h.op0))
        u, v, w = (np.random.default_rng(22 + a).standard_normal(shape).astype(F32) for a in range(3))
        rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
        h.rhs_operator((dev(u), dev(v), dev(w)), dev(ff), rhs, 1.0 / 240.0, 1000.0)
        h.build_coarse()
        P = dev(p0)
        h.w_cycle(P, rhs)
        levels = oracle.Levels(shape)
        q = p0.copy()
        orhs = oracle.pressure_rhs(u, v, w, ff, dx, 1.0 / 240.0, 1000.0, shape)
        levels.w_cycle(q, orhs, ff, oracle.build_finest_operator(ff, shape), dx)
        assert np.array_equal(host(P), q)
    finally:
        backend.lib.clb_mg_set_option(0, 1)
        backend.lib.clb_mg_set_option(1, 1)
        backend.lib.clb_mg_set_option(2, 1)


@pytest.mark.parametrize("cluster", [1, 0])
@pytest.mark.parametrize("shape", [(66, 66, 66), (70, 66, 61), (130, 96, 100)])
def test_scaled_prolongation_matches_oracle(backend, oracle, shape, cluster):
    """W-cycles whose prolonged corrections are scaled (clb_mg_hierarchy.prolong_scale = 1.7) equal the
    oracle's bit for bit, through the cluster visit and level by level; scale 1 is the reference."""
    dx = F32(1.0 / shape[0])
    ff, b, p0 = random_system(shape, 25)
    backend.lib.clb_mg_set_option(2, cluster)
    try:
        h = multigrid.MultigridHierarchy(backend, shape, float(dx))
        u, v, w = (np.random.default_rng(26 + a).standard_normal(shape).astype(F32) for a in range(3))
        rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
        h.rhs_operator((dev(u), dev(v), dev(w)), dev(ff), rhs, 1.0 / 240.0, 1000.0)
        h.build_coarse()
        orhs = oracle.pressure_rhs(u, v, w, ff, dx, 1.0 / 240.0, 1000.0, shape)
        op = oracle.build_finest_operator(ff, shape)
        for scale, cs, k in ((1.7, None, 4), (1.0, None, 4), (1.8, (1, 0), 0), (1.0, (2, 1), 3)):
            P = dev(p0)
            h.w_cycle(P, rhs, pre_smooth=1, post_smooth=1, coarse_iterations=k, prolong_scale=scale, coarse_smooth=cs)
            q = p0.copy()
            oracle.Levels(shape).w_cycle(q, orhs, ff, op, dx, pre=1, post=1, coarse=k, prolong_scale=scale,
                                         pre_coarse=-1 if cs is None else cs[0], post_coarse=-1 if cs is None else cs[1])
            assert np.array_equal(host(P), q), (scale, cs)
    finally:
        backend.lib.clb_mg_set_option(2, 1)
    assert backend.device_error() == 0


def test_programmatic_launch_changes_nothing(backend):
    """Tolerance-mode solves (flexible CG, CUDA graphs) give bit-identical FP64 pressures and cycle
    counts with programmatic dependent launch on and off."""
    shape = (96, 80, 72)
    dx = 1.0 / 96
    ff, _, _ = random_system(shape, 31)
    rng = np.random.default_rng(32)
    vel = [dev(rng.standard_normal(shape).astype(F32)) for _ in range(3)]
    results = {}
    try:
        for pdl in (0, 1):
            backend.lib.clb_mg_set_option(1, pdl)
            ps = pressure_solve.PressureSolver(backend, shape, dx, autotune=False)
            p = torch.zeros(shape, dtype=torch.float32, device="cuda")
            stats = [ps.solve(vel, dev(ff), p, 1.0 / 240.0, 1000.0, tol=1e-6) for _ in range(3)]
            assert all(st.rel_residual <= 1e-6 for st in stats)
            results[pdl] = (host(ps.pressure64), host(p), [st.cycles for st in stats])
    finally:
        backend.lib.clb_mg_set_option(1, 1)
    assert np.array_equal(results[0][0], results[1][0])
    assert np.array_equal(results[0][1], results[1][1])
    assert results[0][2] == results[1][2]
    assert backend.device_error() == 0


@pytest.mark.parametrize("iterations", [1, 3])
def test_fused_smoothing_odd_iterations(backend, oracle, iterations):
    shape, dx = (40, 36, 44), F32(1.0 / 40)
    ff, b, p0 = random_system(shape, 23)
    h = multigrid.MultigridHierarchy(backend, shape, float(dx))
    u, v, w = (np.random.default_rng(24 + a).standard_normal(shape).astype(F32) for a in range(3))
    rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
    h.rhs_operator((dev(u), dev(v), dev(w)), dev(ff), rhs, 1.0 / 240.0, 1000.0)
    assert h.alt[0] is not None
    P = dev(p0)
    h.smooth(0, iterations, P, rhs)
    orhs = oracle.pressure_rhs(u, v, w, ff, dx, 1.0 / 240.0, 1000.0, shape)
    oops = oracle.build_finest_operator(ff, shape)
    q = p0.copy()
    for _ in range(iterations):
        for parity in (0, 1):
            oracle.lib().orc_rbgs_step_f32(q, orhs, ff, *oops, dx, parity, *shape)
    assert np.array_equal(host(P), q)


@pytest.mark.parametrize("kind", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("shape", [(40, 36, 44), (33, 33, 33)])
def test_every_sweep_kind_matches_oracle(backend, oracle, shape, kind):
    dx = F32(1.0 / shape[0])
    ff, b, p0 = random_system(shape, 25)
    h = multigrid.MultigridHierarchy(backend, shape, float(dx), fused_min_cells=1)
    for level in range(h.levels):
        h.set_sweep(level, kind)
    u, v, w = (np.random.default_rng(26 + a).standard_normal(shape).astype(F32) for a in range(3))
    rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
    h.rhs_operator((dev(u), dev(v), dev(w)), dev(ff), rhs, 1.0 / 240.0, 1000.0)
    h.build_coarse()
    orhs = oracle.pressure_rhs(u, v, w, ff, dx, 1.0 / 240.0, 1000.0, shape)
    oops = oracle.build_finest_operator(ff, shape)
    P = dev(p0)
    h.smooth(0, 3, P, rhs)
    q = p0.copy()
    for _ in range(3):
        for parity in (0, 1):
            oracle.lib().orc_rbgs_step_f32(q, orhs, ff, *oops, dx, parity, *shape)
    assert np.array_equal(host(P), q)
    h.w_cycle(P, rhs)
    oracle.Levels(shape).w_cycle(q, orhs, ff, oops, dx)
    assert np.array_equal(host(P), q)


def test_revoxelising_a_static_collider_every_step_changes_nothing(backend):
    s = scenes.collider_pool(32, seed=9, subdivisions=2)
    sims = []
    for revox in (False, True):
        opts = solver.StepOptions(flip_ratio=0.95, num_vcycles=1, gravity=s.gravity, use_graph=False, revoxelise=revox)
        sims.append(solver.scene_solver(backend, s, opts))
    assert sims[1].colliders and int(sims[1].obstacle.sum()) > 0
    mask0 = host(sims[1].obstacle).copy()
    for _ in range(3):
        for sim in sims:
            sim.step()
        assert np.array_equal(host(sims[1].obstacle), mask0)
        assert np.array_equal(sims[0].positions(), sims[1].positions())
        assert np.array_equal(host(sims[0].pressure), host(sims[1].pressure))



@pytest.mark.parametrize("smooth", [(2, 4), (1, 1)])
def test_steps_with_fewer_coarse_iterations(backend, smooth):
    """Tolerance-mode steps with 4 instead of the reference's 64 coarsest-level iterations in the
    W-cycle preconditioner (and with fewer smoothing sweeps) reach the tolerance every step in about as
    many cycles."""
    s = scenes.block(48)
    pos, vel = scenes.seed_particles(s)
    totals = {}
    for k in (64, 4):
        opts = solver.StepOptions(flip_ratio=0.95, tol=1e-6, gravity=s.gravity, coarse_iterations=k,
                                  pre_smooth=smooth[0], post_smooth=smooth[1])
        sim = solver.FlipSolver(backend, s.grid_shape, s.dx, pos, vel, dt=s.dt, options=opts)
        stats = [sim.step() for _ in range(4)]
        assert all(st.rel_residual <= 1e-6 for st in stats)
        assert sim.pressure_solver.coarse_iterations == k
        assert (sim.pressure_solver.pre_smooth, sim.pressure_solver.post_smooth) == smooth
        totals[k] = sum(st.cycles for st in stats)
    assert totals[4] <= totals[64] + 4, totals
    assert backend.device_error() == 0


def corner_block_system(shape, seed):
    """A liquid block in one corner (most tiles hold no fluid) and a random right-hand side."""
    rng = np.random.default_rng(seed)
    ff = np.zeros(shape, F32)
    nx, ny, nz = shape
    ff[1 : nx // 2, 1 : (7 * ny) // 10, 1 : nz // 2] = 1.0
    ff[rng.random(shape) < 0.03] = 0
    return ff


@pytest.mark.parametrize("shape", [(66, 70, 68), (66, 66, 66), (40, 36, 44)])
def test_fluid_tile_w_cycle_matches_oracle(backend, oracle, shape):
    """W-cycles that visit only the tiles holding fluid (level 0 included: a zero correction) give the
    reference's values, and the same values as with the tile lists switched off."""
    dx = F32(1.0 / shape[0])
    ff = corner_block_system(shape, 41)
    u, v, w = (np.random.default_rng(42 + a).standard_normal(shape).astype(F32) for a in range(3))
    orhs = oracle.pressure_rhs(u, v, w, ff, dx, 1.0 / 240.0, 1000.0, shape)
    oops = oracle.build_finest_operator(ff, shape)
    results = {}
    for tiles in (True, False):
        h = multigrid.MultigridHierarchy(backend, shape, float(dx), fluid_tiles=tiles)
        rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
        h.rhs_operator((dev(u), dev(v), dev(w)), dev(ff), rhs, 1.0 / 240.0, 1000.0)
        h.build_coarse()
        if tiles:
            counts = h.tile_counts.cpu().numpy()[: h.levels]
            assert 0 < counts[0] < int(backend.lib.clb_mg_tile_capacity(*shape, 1))
        P = torch.zeros(shape, dtype=torch.float32, device="cuda")
        for _ in range(2):
            h.w_cycle(P, rhs, x_zero_outside=True, coarse_iterations=8)
        results[tiles] = host(P)
    q = np.zeros(shape, F32)
    levels = oracle.Levels(shape)
    for _ in range(2):
        levels.w_cycle(q, orhs, ff, oops, dx, coarse=8)
    assert np.array_equal(results[True], q)
    assert np.array_equal(results[False], q)
    assert backend.device_error() == 0


@pytest.mark.parametrize("shape,pre", [((66, 70, 68), 1), ((40, 36, 44), 2), ((40, 36, 44), 0)])
def test_w_cycle_from_zero_ignores_the_previous_correction(backend, oracle, shape, pre):
    """A W-cycle told that the correction starts from zero (x_from_zero: its first level-0 sweep ignores
    x, or x is zeroed when no sweep comes first) gives the reference's W-cycle from a zero x, although
    the buffer still holds a previous correction at the fluid cells."""
    dx = F32(1.0 / shape[0])
    ff = corner_block_system(shape, 43)
    u, v, w = (np.random.default_rng(52 + a).standard_normal(shape).astype(F32) for a in range(3))
    orhs = oracle.pressure_rhs(u, v, w, ff, dx, 1.0 / 240.0, 1000.0, shape)
    oops = oracle.build_finest_operator(ff, shape)
    h = multigrid.MultigridHierarchy(backend, shape, float(dx))
    rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
    h.rhs_operator((dev(u), dev(v), dev(w)), dev(ff), rhs, 1.0 / 240.0, 1000.0)
    h.build_coarse()
    P = torch.zeros(shape, dtype=torch.float32, device="cuda")
    h.w_cycle(P, rhs, pre_smooth=pre, coarse_iterations=8, x_zero_outside=True)  # a previous correction
    assert P.abs().max() > 0
    h.w_cycle(P, rhs, pre_smooth=pre, coarse_iterations=8, x_from_zero=True)
    q = np.zeros(shape, F32)
    oracle.Levels(shape).w_cycle(q, orhs, ff, oops, dx, pre=pre, coarse=8)
    assert np.array_equal(host(P), q)
    assert backend.device_error() == 0
