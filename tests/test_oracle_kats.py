"""Known-answer tests that pin the oracle (the CPU restatement) to the reference's semantics.

The reference ships no tests or golden vectors and cannot run here, so these answers are derived by
hand (or by an independent numpy/scipy construction) from the reference kernels' definitions, with
inputs chosen so that float32 arithmetic is exact where an exact answer is asserted.
"""

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from continuum_liquid_b200 import scenes


def gidx(i, j, k, ny, nz):
    return (i * ny + j) * nz + k


# ---- binning (particles.cl:3-6, 44-59) -----------------------------------------------------------
def test_bin_keys_known_answers(oracle):
    n, dx = 16, 1.0 / 16.0
    shape = (n, n, n)
    pos = np.array(
        [
            [0.5 * dx, 0.5 * dx, 0.5 * dx],  # s - 0.5 = 0 -> 0
            [1.5 * dx, 2.5 * dx, 3.5 * dx],  # -> (1, 2, 3)
            [0.25 * dx, 1.4375 * dx, 2.0 * dx],  # floor(-0.25) = -1 -> clamp 0; 0.9375 -> 0; 1.5 -> 1
            [15.75 * dx, 14.5 * dx, 13.25 * dx],  # 15.25 -> clamp 14; 14; 12.75 -> 12
        ],
        np.float32,
    )
    expect = [gidx(0, 0, 0, n, n), gidx(1, 2, 3, n, n), gidx(0, 0, 1, n, n), gidx(14, 14, 12, n, n)]
    assert oracle.bin_keys(pos, dx, shape).tolist() == expect
    counts = oracle.count_particles(pos, dx, shape)
    assert counts.sum() == 4 and counts[expect[0]] == 1 and counts[expect[3]] == 1


@pytest.mark.parametrize("size", [0, 1, 7, 511, 512, 513, 4097, 262151])
def test_scan_equals_exclusive_cumsum(oracle, size):
    rng = np.random.default_rng(size)
    values = rng.integers(0, 20, size).astype(np.int32)
    out, total = oracle.exclusive_scan(values)
    expect = np.concatenate([[0], np.cumsum(values)[:-1]]).astype(np.int32) if size else values
    assert np.array_equal(out, expect)
    assert total == int(values.sum())


def test_sort_is_stable_permutation(oracle):
    rng = np.random.default_rng(3)
    n, dx = 12, 1.0 / 12.0
    shape = (n, n, n)
    pos = (rng.random((500, 3)) * (n - 2) + 1.0).astype(np.float32) * np.float32(dx)
    vel = np.arange(1500, dtype=np.float32).reshape(500, 3)  # row id encoded in the velocity
    keys = oracle.bin_keys(pos, dx, shape)
    counts = oracle.count_particles(pos, dx, shape)
    offsets, _ = oracle.exclusive_scan(counts)
    pos_s, vel_s, cursors = oracle.sort_particles(pos, vel, offsets, dx, shape)
    ids = (vel_s[:, 0] / 3).astype(np.int64)
    assert sorted(ids.tolist()) == list(range(500))
    assert np.array_equal(cursors, counts)
    assert np.array_equal(ids, np.argsort(keys, kind="stable"))  # bins ascending, input order inside
    assert np.array_equal(pos_s, pos[ids])


# ---- P2G (particles.cl:135-227) ------------------------------------------------------------------
def test_p2g_single_particle_known_answer(oracle):
    n, dx = 12, 1.0 / 8.0  # inv_dx = 8 exactly
    shape = (n, n, n)
    s = np.array([5.25, 6.75, 4.5])
    pos = (s * dx).astype(np.float32)[None]
    vel = np.array([[0.5, -0.25, 2.0]], np.float32)  # powers of two: (w*v)/w is exact
    _, _, u, v, w, ff, _, _ = oracle.particle_to_grid(pos, vel, dx, shape)
    face = {"u": (1.0, 0.5, 0.5), "v": (0.5, 1.0, 0.5), "w": (0.5, 0.5, 1.0)}
    for name, field, value in (("u", u, 0.5), ("v", v, -0.25), ("w", w, 2.0)):
        expect = np.zeros(shape, np.float32)
        off = face[name]
        for i in range(n):
            for j in range(n):
                for k in range(n):
                    d = np.abs(s - (np.array([i, j, k]) + off))
                    if np.all(d < 1.0):
                        expect[i, j, k] = value
        assert np.array_equal(field, expect), name
    expect_ff = np.zeros(shape, np.float32)
    expect_ff[5, 6, 4] = 0.125  # trunc(s) = (5, 6, 4); ff = count / 8
    assert np.array_equal(ff, expect_ff)


def test_p2g_two_particles_weighted_average(oracle):
    n, dx = 10, 1.0 / 8.0
    shape = (n, n, n)
    s = np.array([[4.25, 4.5, 4.5], [4.75, 4.5, 4.5]])
    pos = (s * dx).astype(np.float32)
    vel = np.array([[1.0, 0, 0], [3.0, 0, 0]], np.float32)
    _, _, u, _, _, ff, _, _ = oracle.particle_to_grid(pos, vel, dx, shape)
    # u face of cell (4,4,4) sits at (5, 4.5, 4.5): tent weights 0.25 and 0.75
    assert u[4, 4, 4] == pytest.approx((0.25 * 1 + 0.75 * 3) / (0.25 + 0.75), rel=1e-7)
    # face of cell (3,4,4) at (4, 4.5, 4.5): weights 0.75 and 0.25
    assert u[3, 4, 4] == pytest.approx((0.75 * 1 + 0.25 * 3) / 1.0, rel=1e-7)
    assert ff[4, 4, 4] == 0.25


# ---- G2P, advection, particle boundaries ---------------------------------------------------------
def test_g2p_linear_field_exact(oracle):
    n, dx = 12, 1.0 / 8.0
    shape = (n, n, n)
    I, J, K = np.meshgrid(*(np.arange(n, dtype=np.float32),) * 3, indexing="ij")
    lin = (I + 2 * J + 3 * K).astype(np.float32)
    zero = np.zeros(shape, np.float32)
    s = np.array([5.25, 6.75, 4.5])
    pos = (s * dx).astype(np.float32)[None]
    vel = np.zeros((1, 3), np.float32)
    out = oracle.grid_to_particle(vel, pos, (lin, lin, lin), (zero, zero, zero), dx, shape)
    # u samples at grid coordinates s - (1, 0.5, 0.5), v at s - (0.5, 1, 0.5), w at s - (0.5, 0.5, 1)
    for a, off in enumerate([(1, 0.5, 0.5), (0.5, 1, 0.5), (0.5, 0.5, 1)]):
        g = s - np.array(off)
        assert out[0, a] == g[0] + 2 * g[1] + 3 * g[2]
    # FLIP keeps the increment only: with old == new the velocity is unchanged
    out2 = oracle.grid_to_particle(np.ones((1, 3), np.float32), pos, (lin,) * 3, (lin,) * 3, dx, shape)
    assert np.array_equal(out2, np.ones((1, 3), np.float32))


def test_advect_and_domain_reflection(oracle):
    n, dx = 16, 1.0 / 16.0
    shape = (n, n, n)
    pos = np.array([[0.5, 0.5, 0.5]], np.float32)
    vel = np.array([[1.0, -2.0, 0.25]], np.float32)
    out = oracle.advect(pos, vel, 0.125)
    assert np.array_equal(out, np.array([[0.625, 0.25, 0.53125]], np.float32))
    lower = np.float32(1.001 * dx)
    upper = np.float32((n - 1.001) * dx)
    p = np.array([[lower - np.float32(0.01), 0.5, upper + np.float32(0.01)]], np.float32)
    v = np.array([[-1.0, 3.0, 2.0]], np.float32)
    p2, v2 = oracle.particle_domain_bc(p, v, dx, shape)
    assert p2[0, 0] == np.float32(np.float32(2.0) * lower - p[0, 0])
    assert p2[0, 2] == np.float32(np.float32(2.0) * upper - p[0, 2])
    assert v2.tolist() == [[0.0, 3.0, 0.0]]


def test_particle_obstacle_pushout(oracle):
    n, dx = 8, 1.0 / 8.0
    shape = (n, n, n)
    obstacle = np.zeros(shape, np.uint8)
    obstacle[4, 4, 4] = 1
    prev = (np.array([[3.9, 4.5, 4.5]]) * dx).astype(np.float32)
    pos = (np.array([[4.25, 4.5, 4.5]]) * dx).astype(np.float32)
    vel = np.array([[1.0, 0.5, 0.0]], np.float32)
    p2, v2 = oracle.particle_obstacle_bc(pos, prev, vel, obstacle, dx, shape)
    # entered through the -x face: normal (-1,0,0); inward normal velocity removed; reflected about x = 4 dx
    assert v2.tolist() == [[0.0, 0.5, 0.0]]
    assert p2[0, 0] == np.float32(np.float32(2.0) * np.float32(4 * dx) - pos[0, 0])
    assert p2[0, 1] == pos[0, 1] and p2[0, 2] == pos[0, 2]


# ---- grid kernels -------------------------------------------------------------------------------
def test_pressure_rhs_linear_divergence(oracle):
    n, dx = 10, 1.0 / 16.0
    shape = (n, n, n)
    I, J, K = np.meshgrid(*(np.arange(n, dtype=np.float32),) * 3, indexing="ij")
    ff = np.zeros(shape, np.float32)
    ff[1:-1, 1:-1, 1:-1] = 1.0
    ff[2, 2, 2] = 0.0
    rhs = oracle.pressure_rhs(I, 2 * J, 4 * K, ff, dx, 1.0 / 240.0, 1000.0, shape)
    expect = np.zeros(shape, np.float32)
    expect[1:-1, 1:-1, 1:-1] = np.float32(1000.0 / (1.0 / 240.0)) * np.float32(7 * 16)
    expect[2, 2, 2] = 0.0
    assert np.array_equal(rhs, expect)


def test_grid_domain_bc_walls_and_ghosts(oracle):
    n = 8
    shape = (n, n, n)
    rng = np.random.default_rng(1)
    u, v, w = (rng.standard_normal(shape).astype(np.float32) for _ in range(3))
    u2, v2, w2 = oracle.grid_domain_bc(u, v, w, shape)
    assert not u2[0].any() and not u2[n - 2 :].any()
    assert not v2[:, 0].any() and not v2[:, n - 2 :].any()
    assert not w2[:, :, 0].any() and not w2[:, :, n - 2 :].any()
    assert np.array_equal(u2[1 : n - 2, 1:-1, 1:-1], u[1 : n - 2, 1:-1, 1:-1])
    # a y-ghost copies u from the clamped interior cell
    assert u2[3, 0, 4] == u[3, 1, 4] and u2[3, n - 1, 4] == u[3, n - 2, 4]


def test_neumann_ghost_copy(oracle):
    n = 6
    shape = (n, n, n)
    p = np.random.default_rng(2).standard_normal(shape).astype(np.float32)
    q = oracle.neumann_domain_bc(p, shape)
    idx = np.clip(np.arange(n), 1, n - 2)
    expect = p[np.ix_(idx, idx, idx)]
    assert np.array_equal(q, expect)


def test_update_velocity_gravity_only(oracle):
    n, dx, dt = 8, 1.0 / 8.0, 0.25
    shape = (n, n, n)
    ff = np.zeros(shape, np.float32)
    ff[3, 3, 3] = 0.5
    zero = np.zeros(shape, np.float32)
    u, v, w = oracle.update_velocity(zero, zero, zero, ff, (0.0, -8.0, 0.0), (0.0, 0.0, 0.0), 1000.0, 0.0, dx, dt,
                                     shape)
    assert v[3, 3, 3] == -2.0 and np.count_nonzero(v) == 1 and not u.any() and not w.any()


# ---- voxelisation (voxelise_mesh.cl) -------------------------------------------------------------
def cube_triangles(lo, hi):
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    c = np.array([[lo[0] if b & 1 == 0 else hi[0], lo[1] if b & 2 == 0 else hi[1], lo[2] if b & 4 == 0 else hi[2]]
                  for b in range(8)])
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    tris = []
    for a, b, cc, d in quads:
        tris += [(c[a], c[b], c[cc]), (c[a], c[cc], c[d])]
    return np.asarray(tris, np.float32)


def test_voxelise_cube_known_answer(oracle):
    n, delta = 24, 1.0 / 24.0
    shape = (n, n, n)
    origin = (-0.5, -0.5, 0.0)
    lo = np.array([-0.2013, -0.1777, 0.3031])
    hi = np.array([0.1991, 0.2207, 0.6969])
    mask = oracle.voxelise(cube_triangles(lo, hi), shape, delta, origin)
    centres = [origin[a] + (np.arange(n) + 0.5) * delta for a in range(3)]
    X, Y, Z = np.meshgrid(*centres, indexing="ij")
    inside = (X > lo[0]) & (X < hi[0]) & (Y > lo[1]) & (Y < hi[1]) & (Z > lo[2]) & (Z < hi[2])
    inside[[0, -1], :, :] = inside[:, [0, -1], :] = inside[:, :, [0, -1]] = False  # ghosts are never set
    assert np.array_equal(mask.astype(bool), inside)


def test_voxelise_icosphere_inside_outside(oracle):
    n, delta = 32, 1.0 / 32.0
    shape = (n, n, n)
    origin = (-0.5, -0.5, 0.0)
    centre = np.array([0.03, -0.02, 0.51])
    r = 0.3
    mask = oracle.voxelise(scenes.icosphere(2, r, centre), shape, delta, origin)
    centres = [origin[a] + (np.arange(n) + 0.5) * delta for a in range(3)]
    X, Y, Z = np.meshgrid(*centres, indexing="ij")
    d = np.sqrt((X - centre[0]) ** 2 + (Y - centre[1]) ** 2 + (Z - centre[2]) ** 2)
    # subdivision-2 facets lie within ~1.5% of r of the sphere
    assert mask[d < 0.95 * r].all()
    assert not mask[d > 1.01 * r].any()


# ---- multigrid (multigrid.cl / multigrid.py) ------------------------------------------------------
def liquid_mask(n, seed):
    rng = np.random.default_rng(seed)
    m = np.zeros((n, n, n), np.float32)
    m[1:-1, 1 : n // 2 + 1, 1:-1] = 1.0  # liquid below mid-height, air above (Dirichlet p = 0)
    holes = rng.random((n, n, n)) < 0.1
    m[holes] = 0.0
    m[1:-1, 1:-1, 1:-1][m[1:-1, 1:-1, 1:-1] == 0] *= 1
    return m


def dense_operator(mask, dx):
    """A from the reference definitions (multigrid.cl:3-88), built independently in numpy, as a
    sparse matrix over interior fluid cells: (A p)_c = (sum_nb w p_nb - diag_c p_c) / dx^2."""
    n = mask.shape[0]
    cells = [(i, j, k) for i in range(1, n - 1) for j in range(1, n - 1) for k in range(1, n - 1) if mask[i, j, k] > 0]
    index = {c: t for t, c in enumerate(cells)}
    rows, cols, vals = [], [], []
    for (i, j, k), t in index.items():
        diag = 6 - (i == 1) - (i == n - 2) - (j == 1) - (j == n - 2) - (k == 1) - (k == n - 2)
        rows.append(t)
        cols.append(t)
        vals.append(-diag / dx**2)
        for di, dj, dk in [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]:
            nb = (i + di, j + dj, k + dk)
            if nb in index:
                rows.append(t)
                cols.append(index[nb])
                vals.append(1.0 / dx**2)
    N = len(cells)
    return sp.csr_matrix((vals, (rows, cols)), shape=(N, N)), cells


def test_finest_operator_matches_definition(oracle):
    n, dx = 10, 0.125
    mask = liquid_mask(n, 4)
    d, wx, wy, wz = oracle.build_finest_operator(mask, (n, n, n))
    A, cells = dense_operator(mask, dx)
    # rebuild the matrix from the oracle's arrays and compare
    index = {c: t for t, c in enumerate(cells)}
    B = sp.lil_matrix(A.shape)
    for (i, j, k), t in index.items():
        B[t, t] = -d[i, j, k] / dx**2
        for axis, wgt in enumerate((wx, wy, wz)):
            for sgn in (1, -1):
                nb = [i, j, k]
                nb[axis] += sgn
                nb = tuple(nb)
                w_ = wgt[i, j, k] if sgn == 1 else wgt[nb]
                if nb in index and w_ != 0:
                    B[t, index[nb]] = w_ / dx**2
    assert abs(A - B.tocsr()).max() == 0


def test_restriction_is_galerkin(oracle):
    """Coarse operator and right-hand side of restrict_residual equal P^T A P and P^T r for the
    piecewise-constant aggregation P (coarse cell I <- fine cells 1 + 2(I-1) + {0,1})."""
    n, dx = 12, 0.125
    shape = (n, n, n)
    mask = liquid_mask(n, 5)
    rng = np.random.default_rng(6)
    p = (rng.standard_normal(shape) * (mask > 0)).astype(np.float32)
    b = (rng.standard_normal(shape) * (mask > 0)).astype(np.float32)
    op = oracle.build_finest_operator(mask, shape)
    cshape = tuple(oracle.coarse_grid_size(s) for s in shape)
    carr = [np.zeros(cshape, np.float32) for _ in range(7)]
    oracle.lib().orc_restrict_residual_f32(p, b, mask, *op, *carr, np.float32(dx), *shape, *cshape)
    cp, cb, cm, cd, cwx, cwy, cwz = carr
    A, cells = dense_operator(mask, dx)
    agg = {}
    for t, (i, j, k) in enumerate(cells):
        agg.setdefault(((i - 1) // 2 + 1, (j - 1) // 2 + 1, (k - 1) // 2 + 1), []).append(t)
    coarse = sorted(agg)
    cidx = {c: t for t, c in enumerate(coarse)}
    P = sp.lil_matrix((len(cells), len(coarse)))
    for c_, members in agg.items():
        for t in members:
            P[t, cidx[c_]] = 1.0
    P = P.tocsr()
    Ac = (P.T @ A @ P).toarray() * dx**2
    pv = np.array([p[c] for c in cells], np.float64)
    bv = np.array([b[c] for c in cells], np.float64)
    r = bv - A @ pv
    rc = P.T @ r
    assert not cp.any()
    for c_, t in cidx.items():
        assert cm[c_] == 1.0
        assert cd[c_] == pytest.approx(-Ac[t, t], abs=1e-9)
        for axis, wgt in enumerate((cwx, cwy, cwz)):
            nb = list(c_)
            nb[axis] += 1
            nb = tuple(nb)
            expect = Ac[t, cidx[nb]] if nb in cidx else 0.0
            assert wgt[c_] == pytest.approx(expect, abs=1e-9)
        assert cb[c_] == pytest.approx(rc[t], rel=2e-4, abs=1e-2 * np.abs(rc).max() * 1e-3)
    assert int(cm.sum()) == len(coarse)


def test_fp64_multigrid_solves_the_linear_system(oracle):
    """The oracle's FP64 W-cycle converges to the solution of A p = b from an independent sparse
    direct solve."""
    n, dx = 14, 1.0 / 14.0
    shape = (n, n, n)
    mask = liquid_mask(n, 7)
    rng = np.random.default_rng(8)
    b = (rng.standard_normal(shape) * (mask > 0)).astype(np.float32)
    p, history = oracle.fp64_pressure_solve(b, mask, shape, dx, tol=1e-12, max_cycles=300)
    assert history[-1] <= 1e-12
    assert all(h1 < h0 for h0, h1 in zip(history, history[1:]))
    A, cells = dense_operator(mask, dx)
    x = spla.spsolve(A.tocsc(), np.array([b[c] for c in cells], np.float64))
    got = np.array([p[c] for c in cells])
    assert np.abs(got - x).max() <= 1e-9 * np.abs(x).max()


def test_float32_w_cycle_contracts(oracle):
    n, dx = 18, 1.0 / 18.0
    shape = (n, n, n)
    mask = liquid_mask(n, 9)
    rng = np.random.default_rng(10)
    b = (rng.standard_normal(shape) * (mask > 0)).astype(np.float32)
    op = oracle.build_finest_operator(mask, shape)
    levels = oracle.Levels(shape)
    p = np.zeros(shape, np.float32)
    rels = [oracle.relative_residual(p, b, mask, op, dx)]
    for _ in range(6):
        levels.w_cycle(p, b, mask, op, dx)
        rels.append(oracle.relative_residual(p, b, mask, op, dx))
    assert all(r1 < 0.8 * r0 for r0, r1 in zip(rels, rels[1:]))
    assert (mask <= 0).sum() and not p[mask <= 0].any()  # air and ghost pressure held at 0


def test_operator_apply_matches_dense_operator(oracle):
    n, dx = 12, 1.0 / 12.0
    shape = (n, n, n)
    mask = liquid_mask(n, 11)
    rng = np.random.default_rng(12)
    p = rng.standard_normal(shape) * (mask > 0)
    op = oracle.build_finest_operator(mask.astype(np.float64), shape, np.float64)
    got, fluid = oracle.apply_operator64(p, mask, op, dx)
    A, cells = dense_operator(mask, dx)
    x = np.array([p[c] for c in cells])
    want = A @ x
    assert fluid.sum() == len(cells)
    np.testing.assert_allclose([got[c] for c in cells], want, rtol=1e-12, atol=1e-9 * np.abs(want).max())


def test_fcg_restatement(oracle):
    """The FCG restatement reports the true FP64 residual of its pressure, reaches the tolerance in
    fewer W-cycles than refinement, and with flexible=False is exactly W-cycles on the pressure."""
    n, dx = 18, np.float32(1.0 / 18.0)
    shape = (n, n, n)
    mask = liquid_mask(n, 9)
    rng = np.random.default_rng(13)
    b = (rng.standard_normal(shape) * (mask > 0)).astype(np.float32)
    x, hist = oracle.fcg_solve(b, mask, shape, dx, tol=1e-8, max_cycles=60)
    _, hist_ref = oracle.fcg_solve(b, mask, shape, dx, tol=1e-8, max_cycles=60, flexible=False)
    op64 = oracle.build_finest_operator(mask.astype(np.float64), shape, np.float64)
    assert hist[-1] <= 1e-8 and hist_ref[-1] <= 1e-8
    assert oracle.relative_residual(x, b.astype(np.float64), mask.astype(np.float64), op64, float(dx)) == \
        pytest.approx(hist[-1], rel=1e-6)
    assert len(hist) < len(hist_ref)
    # refinement from zero: its first iterate is one FP32 W-cycle on the pressure
    x1, _ = oracle.fcg_solve(b, mask, shape, dx, tol=0.0, max_cycles=1, flexible=False)
    p = np.zeros(shape, np.float32)
    oracle.Levels(shape).w_cycle(p, b, mask, oracle.build_finest_operator(mask, shape), dx)
    assert np.array_equal(x1, np.where(mask > 0, p, 0).astype(np.float64))


def test_scaled_prolongation(oracle):
    """prolong_scale = 1 is the reference's W-cycle bit for bit; 1.7 over-corrects the piecewise-constant
    prolongation and the FCG restatement needs fewer W-cycles to the same tolerance."""
    n, dx = 34, np.float32(1.0 / 34.0)
    shape = (n, n, n)
    mask = np.zeros(shape, np.float32)
    mask[1:-1, 1 : n // 2 + 1, 1:-1] = 1.0  # a liquid slab under air, no air cells inside it
    rng = np.random.default_rng(15)
    b = (rng.standard_normal(shape) * (mask > 0)).astype(np.float32)
    ops = oracle.build_finest_operator(mask, shape)
    p1, p2 = np.zeros(shape, np.float32), np.zeros(shape, np.float32)
    oracle.Levels(shape).w_cycle(p1, b, mask, ops, dx)
    oracle.Levels(shape).w_cycle(p2, b, mask, ops, dx, prolong_scale=1.0)
    assert np.array_equal(p1, p2)
    _, hist1 = oracle.fcg_solve(b, mask, shape, dx, tol=1e-8, max_cycles=60, coarse_iterations=4, pre_smooth=1,
                                post_smooth=1)
    _, hist17 = oracle.fcg_solve(b, mask, shape, dx, tol=1e-8, max_cycles=60, coarse_iterations=4, pre_smooth=1,
                                 post_smooth=1, prolong_scale=1.7)
    assert hist1[-1] <= 1e-8 and hist17[-1] <= 1e-8
    assert len(hist17) + 4 <= len(hist1)  # 13 against 19 W-cycles


def test_coarse_level_smoothing_counts(oracle):
    """Coarse-level counts equal to the W-cycle's give the reference's W-cycle bit for bit; without the
    coarse levels' post-smoothing and with the scaled prolongation the FCG restatement still converges."""
    n, dx = 34, np.float32(1.0 / 34.0)
    shape = (n, n, n)
    mask = np.zeros(shape, np.float32)
    mask[1:-1, 1 : n // 2 + 1, 1:-1] = 1.0
    b = (np.random.default_rng(16).standard_normal(shape) * (mask > 0)).astype(np.float32)
    ops = oracle.build_finest_operator(mask, shape)
    p1, p2 = np.zeros(shape, np.float32), np.zeros(shape, np.float32)
    oracle.Levels(shape).w_cycle(p1, b, mask, ops, dx, pre=2, post=4, coarse=8)
    oracle.Levels(shape).w_cycle(p2, b, mask, ops, dx, pre=2, post=4, coarse=8, pre_coarse=2, post_coarse=4)
    assert np.array_equal(p1, p2)
    p3 = np.zeros(shape, np.float32)
    oracle.Levels(shape).w_cycle(p3, b, mask, ops, dx, pre=2, post=4, coarse=8, pre_coarse=1, post_coarse=0)
    assert not np.array_equal(p1, p3)
    _, hist = oracle.fcg_solve(b, mask, shape, dx, tol=1e-8, max_cycles=60, coarse_iterations=0, pre_smooth=1,
                               post_smooth=1, prolong_scale=1.8, coarse_smooth=(1, 0))
    assert hist[-1] <= 1e-8 and len(hist) <= 30


def test_fcg_with_fewer_coarse_iterations(oracle):
    """The FCG restatement still converges with a weak coarsest-level solve in its W-cycle."""
    n, dx = 18, np.float32(1.0 / 18.0)
    shape = (n, n, n)
    mask = liquid_mask(n, 9)
    rng = np.random.default_rng(14)
    b = (rng.standard_normal(shape) * (mask > 0)).astype(np.float32)
    _, hist64 = oracle.fcg_solve(b, mask, shape, dx, tol=1e-8, max_cycles=60)
    _, hist4 = oracle.fcg_solve(b, mask, shape, dx, tol=1e-8, max_cycles=60, coarse_iterations=4)
    assert hist4[-1] <= 1e-8
    assert len(hist4) <= len(hist64) + 3


def test_single_visit_levels(oracle):
    """The single-visit variant of the W-cycle: from a level past the coarsest it is the reference's
    W-cycle; from the coarsest it runs one coarse solve per visit of the level above, which is the
    reference W-cycle with half the coarsest-level iterations there when pre-smoothing is 0."""
    shape = (34, 30, 38)
    rng = np.random.default_rng(11)
    ff = np.zeros(shape, np.float32)
    ff[1:-1, 1:20, 1:-1] = 1.0
    ff[rng.random(shape) < 0.05] = 0
    b = (rng.standard_normal(shape) * (ff > 0)).astype(np.float32)
    dx = np.float32(1.0 / 34)
    ops = oracle.build_finest_operator(ff, shape)
    levels = oracle.Levels(shape)
    n = len(levels.shapes)
    results = {}
    for single in (0, n, n - 1):
        q = np.zeros(shape, np.float32)
        oracle.Levels(shape).w_cycle(q, b, ff, ops, dx, pre=0, post=2, coarse=8, single_from=single)
        results[single] = q
    assert np.array_equal(results[0], results[n])
    q = np.zeros(shape, np.float32)
    oracle.Levels(shape).w_cycle(q, b, ff, ops, dx, pre=0, post=2, coarse=4)
    assert np.array_equal(results[n - 1], q)
