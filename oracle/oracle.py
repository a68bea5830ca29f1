"""ORACLE -- test infrastructure only; never imported by the product package.

Python side of the CPU restatement of Continuum Liquid's FLIP solver: a ctypes binding of
liboracle.so (flip_oracle.cpp, one function per reference OpenCL kernel) and a numpy restatement
of the host orchestration in Solver/Kernel/solver.py:243-529, particles.py:73-171,
multigrid.py:18-187 and pressure_solve.py:10-85.

Parity status: pinned to the reference itself. The reference ships no tests or golden vectors and
no OpenCL runtime exists here, so oracle/reference_run.py runs the reference's own host code and
OpenCL kernels on the CPU (oracle/pyopencl_shim, oracle/ref_build.py -> oracle/_ref/); the bakes it
produced are committed as tests/golden/ref_*, and tests/test_reference_golden.py checks this
restatement against them bit for bit (every frame and every intermediate of the first step).
Hand-derived known-answer tests (tests/test_oracle_kats.py) check it as well.
"""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
LIBRARY = ORACLE_DIR / "liboracle.so"

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_I, _L, _F, _D, _P = ctypes.c_int, ctypes.c_int64, ctypes.c_float, ctypes.c_double, ctypes.c_void_p

_SIGS = {
    "orc_bin_keys": [_f32p, _i32p, _L, _F, _I, _I, _I],
    "orc_count_particles_per_cell": [_f32p, _i32p, _L, _F, _I, _I, _I],
    "orc_scan_blocks_exclusive": [_i32p, _i32p, _i32p, _L, _I],
    "orc_add_scanned_block_offsets": [_i32p, _i32p, _L, _I],
    "orc_exclusive_prefix_sum": [_i32p, _i32p, _L, _I, _P],
    "orc_sort_particles": [_f32p, _f32p, _f32p, _f32p, _i32p, _i32p, _L, _F, _I, _I, _I],
    "orc_particle_to_grid_gather": [_f32p, _f32p, _i32p, _i32p, _f32p, _f32p, _f32p, _f32p, _F, _F, _I, _I, _I, _I],
    "orc_grid_to_particle": [_f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _L, _F, _I, _I, _I, _F],
    "orc_advect_particles": [_f32p, _f32p, _L, _F],
    "orc_voxelise_direction": [_f32p],
    "orc_voxelise_mesh": [_f32p, _u8p, _I, _I, _I, _I, _F, _F, _F, _F],
    "orc_update_velocity": [_f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p] + [_F] * 10 + [_I, _I, _I],
    "orc_grid_domain_bc": [_f32p, _f32p, _f32p, _I, _I, _I],
    "orc_grid_obstacle_bc": [_f32p, _f32p, _f32p, _f32p, _u8p, _I, _I, _I],
    "orc_extrapolate_obstacle_velocity": [_f32p, _f32p, _f32p, _u8p, _I, _I, _I],
    "orc_particle_domain_bc": [_f32p, _f32p, _L, _F, _F, _F, _F],
    "orc_particle_obstacle_bc": [_f32p, _f32p, _f32p, _u8p, _L, _F, _I, _I, _I],
    "orc_pressure_rhs": [_f32p, _f32p, _f32p, _f32p, _f32p, _F, _F, _I, _I, _I],
    "orc_pressure_correction": [_f32p, _f32p, _f32p, _f32p, _F, _F, _I, _I, _I],
    "orc_neumann_domain_bc": [_f32p, _I, _I, _I],
    "orc_build_finest_operator_f32": [_f32p] * 5 + [_I, _I, _I],
    "orc_build_finest_operator_f64": [_f64p] * 5 + [_I, _I, _I],
    "orc_restrict_residual_f32": [_f32p] * 14 + [_F, _I, _I, _I, _I, _I, _I],
    "orc_prolongate_f32": [_f32p, _f32p, _f32p, _I, _I, _I, _I, _I, _I],
    "orc_rbgs_step_f32": [_f32p] * 7 + [_F, _I, _I, _I, _I],
    "orc_coarse_smooth_f32": [_f32p] * 7 + [_F, _I, _I, _I, _I],
    "orc_w_cycle_f32": [_P] * 7 + [_P, _I, _F, _I, _I, _I, _I, _F, _I, _I],
    "orc_w_cycle_f64": [_P] * 7 + [_P, _I, _D, _I, _I, _I, _I, _D, _I, _I],
    "orc_residual_norms_f32": [_f32p] * 7 + [_F, _I, _I, _I, _P, _P],
    "orc_residual_norms_f64": [_f64p] * 7 + [_D, _I, _I, _I, _P, _P],
    "orc_fcg_update": [_f32p, _f32p, _f64p, _f64p, _f32p, _f64p, _f32p, _f64p, _f64p, _f64p, _f64p, _D, _I, _I, _I,
                       _I, _P, _P],
    "orc_grid_obstacle_bc_moving": [_f32p, _f32p, _f32p, _f32p, _u8p, _I, _I, _I, _f32p, _F],
    "orc_extrapolate_obstacle_velocity_moving": [_f32p, _f32p, _f32p, _u8p, _I, _I, _I, _f32p, _F],
    "orc_particle_obstacle_bc_moving": [_f32p, _f32p, _f32p, _u8p, _L, _F, _I, _I, _I, _f32p],
    "orc_num_threads": [],
}


def build() -> Path:
    """Compile liboracle.so with the committed Makefile (gcc, -ffp-contract=off, OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
    return LIBRARY


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            build()
        handle = ctypes.CDLL(str(LIBRARY))
        for name, argtypes in _SIGS.items():
            fn = getattr(handle, name)
            fn.argtypes = argtypes
            fn.restype = _I if name == "orc_num_threads" else None
        _lib = handle
    return _lib


F32 = np.float32


def c(a, dtype=np.float32):
    return np.ascontiguousarray(a, dtype=dtype)


# ---- particles ---------------------------------------------------------------------------------
def bin_keys(pos, dx, shape):
    keys = np.zeros(len(pos), np.int32)
    lib().orc_bin_keys(c(pos), keys, len(pos), F32(1.0 / float(dx)), *shape)
    return keys


def count_particles(pos, dx, shape):
    counts = np.zeros(int(np.prod(shape)), np.int32)
    lib().orc_count_particles_per_cell(c(pos), counts, len(pos), F32(1.0 / float(dx)), *shape)
    return counts


def exclusive_scan(values, L=256):
    values = c(values, np.int32)
    out = np.zeros_like(values)
    total = ctypes.c_int32(0)
    lib().orc_exclusive_prefix_sum(values, out, len(values), L, ctypes.addressof(total))
    return out, int(total.value)


def sort_particles(pos, vel, offsets, dx, shape):
    pos_s, vel_s = np.zeros_like(c(pos)), np.zeros_like(c(vel))
    cursors = np.zeros(int(np.prod(shape)), np.int32)
    lib().orc_sort_particles(c(pos), c(vel), pos_s, vel_s, c(offsets, np.int32), cursors, len(pos), F32(1.0 / float(dx)),
                             *shape)
    return pos_s, vel_s, cursors


def p2g_gather(pos_sorted, vel_sorted, offsets, counts, dx, shape, ppc=8, lanes=8):
    C = int(np.prod(shape))
    u, v, w, ff = (np.zeros(C, np.float32) for _ in range(4))
    lib().orc_particle_to_grid_gather(c(pos_sorted), c(vel_sorted), c(offsets, np.int32), c(counts, np.int32), u, v, w,
                                      ff, F32(1.0 / float(dx)), F32(1.0 / ppc), *shape, lanes)
    return tuple(a.reshape(shape) for a in (u, v, w, ff))


def particle_to_grid(pos, vel, dx, shape, ppc=8):
    """particles.py:73-171: returns (sorted pos, sorted vel, u, v, w, ff, counts, offsets)."""
    counts = count_particles(pos, dx, shape)
    offsets, _ = exclusive_scan(counts)
    pos_s, vel_s, cursors = sort_particles(pos, vel, offsets, dx, shape)
    u, v, w, ff = p2g_gather(pos_s, vel_s, offsets, cursors, dx, shape, ppc)
    return pos_s, vel_s, u, v, w, ff, counts, offsets


def grid_to_particle(vel, pos, cur, old, dx, shape, flip_ratio=1.0):
    vel = c(vel).copy()
    lib().orc_grid_to_particle(vel, c(pos), *(c(a) for a in cur), *(c(a) for a in old), len(pos), F32(1.0 / float(dx)),
                               *shape, F32(flip_ratio))
    return vel


def advect(pos, vel, dt):
    pos = c(pos).copy()
    lib().orc_advect_particles(pos, c(vel), len(pos), F32(dt))
    return pos


def particle_domain_bc(pos, vel, dx, shape):
    pos, vel = c(pos).copy(), c(vel).copy()
    lib().orc_particle_domain_bc(pos, vel, len(pos), F32(1.001 * float(dx)), F32((shape[0] - 1.001) * float(dx)),
                                 F32((shape[1] - 1.001) * float(dx)), F32((shape[2] - 1.001) * float(dx)))
    return pos, vel


def particle_obstacle_bc(pos, prev, vel, obstacle, dx, shape, motion=None):
    pos, vel = c(pos).copy(), c(vel).copy()
    if motion is None:
        lib().orc_particle_obstacle_bc(pos, c(prev), vel, c(obstacle, np.uint8), len(pos), F32(1.0 / float(dx)),
                                       *shape)
    else:
        lib().orc_particle_obstacle_bc_moving(pos, c(prev), vel, c(obstacle, np.uint8), len(pos),
                                              F32(1.0 / float(dx)), *shape, c(motion))
    return pos, vel


# ---- voxelisation ------------------------------------------------------------------------------
def voxelise_direction():
    out = np.zeros(3, np.float32)
    lib().orc_voxelise_direction(out)
    return out


def voxelise(triangles, shape, delta, origin, mask=None):
    mask = np.zeros(shape, np.uint8) if mask is None else c(mask, np.uint8).copy()
    tris = c(triangles).reshape(-1, 9)
    lib().orc_voxelise_mesh(tris, mask, len(tris), *shape, F32(delta), F32(origin[0]), F32(origin[1]),
                            F32(origin[2]))
    return mask


# ---- grid kernels ------------------------------------------------------------------------------
def update_velocity(u, v, w, ff, gravity, force, rho, nu, dx, dt, shape):
    out = [np.zeros(shape, np.float32) for _ in range(3)]
    lib().orc_update_velocity(c(u), c(v), c(w), *out, c(ff), F32(gravity[0]), F32(gravity[1]), F32(gravity[2]),
                              F32(force[0]), F32(force[1]), F32(force[2]), F32(rho), F32(nu), F32(1.0 / (float(dx) * float(dx))),
                              F32(dt), *shape)
    return out


def grid_domain_bc(u, v, w, shape):
    u, v, w = c(u).copy(), c(v).copy(), c(w).copy()
    lib().orc_grid_domain_bc(u, v, w, *shape)
    return u, v, w


def grid_obstacle_bc(u, v, w, ff, obstacle, shape, motion=None, dx=None):
    """boundary_conditions.py:53-79: grid_obstacle_bc then extrapolate_obstacle_velocity. ``motion``
    (9 floats: velocity, angular velocity, pivot in grid-local coordinates; with the cell size ``dx``):
    a moving collider (no counterpart in the reference)."""
    u, v, w, ff = c(u).copy(), c(v).copy(), c(w).copy(), c(ff).copy()
    ob = c(obstacle, np.uint8)
    if motion is None:
        lib().orc_grid_obstacle_bc(u, v, w, ff, ob, *shape)
        lib().orc_extrapolate_obstacle_velocity(u, v, w, ob, *shape)
    else:
        m = c(motion)
        lib().orc_grid_obstacle_bc_moving(u, v, w, ff, ob, *shape, m, F32(dx))
        lib().orc_extrapolate_obstacle_velocity_moving(u, v, w, ob, *shape, m, F32(dx))
    return u, v, w, ff


def pressure_rhs(u, v, w, ff, dx, dt, rho, shape):
    rhs = np.zeros(shape, np.float32)
    lib().orc_pressure_rhs(c(u), c(v), c(w), c(ff), rhs, F32(float(rho) / float(dt)), F32(1.0 / float(dx)), *shape)
    return rhs


def pressure_correction(u, v, w, p, dx, dt, rho, shape):
    u, v, w = c(u).copy(), c(v).copy(), c(w).copy()
    lib().orc_pressure_correction(u, v, w, c(p), F32(float(dt) / float(rho)), F32(1.0 / float(dx)), *shape)
    return u, v, w


def neumann_domain_bc(p, shape):
    p = c(p).copy()
    lib().orc_neumann_domain_bc(p, *shape)
    return p


# ---- multigrid ---------------------------------------------------------------------------------
def coarse_grid_size(n):
    return (max(0, n - 2) + 1) // 2 + 2


def level_shapes(shape, min_size=8):
    out = []
    nx, ny, nz = (coarse_grid_size(s) for s in shape)
    while nx >= min_size and ny >= min_size and nz >= min_size:
        out.append((nx, ny, nz))
        nx, ny, nz = coarse_grid_size(nx), coarse_grid_size(ny), coarse_grid_size(nz)
    return out


def build_finest_operator(mask, shape, dtype=np.float32):
    arrays = [np.zeros(shape, dtype) for _ in range(4)]
    fn = lib().orc_build_finest_operator_f32 if dtype == np.float32 else lib().orc_build_finest_operator_f64
    fn(c(mask, dtype), *arrays, *shape)
    return arrays


class Levels:
    """multigrid.py:18-50 levels (reference layout) plus level 0 in one pointer table."""

    def __init__(self, shape, min_size=8, dtype=np.float32):
        self.dtype = dtype
        self.shapes = [tuple(shape), *level_shapes(shape, min_size)]
        self.p = [None] + [np.zeros(s, dtype) for s in self.shapes[1:]]
        self.b = [None] + [np.zeros(s, dtype) for s in self.shapes[1:]]
        self.m = [None] + [np.zeros(s, dtype) for s in self.shapes[1:]]
        self.ops = [None] + [[np.zeros(s, dtype) for _ in range(4)] for s in self.shapes[1:]]

    def w_cycle(self, p, b, mask, op0, delta, pre=2, post=4, coarse=64, single_from=0, prolong_scale=1.0,
                pre_coarse=-1, post_coarse=-1):
        """multigrid.py:53-187 (C++ recursion over the whole pyramid). single_from > 0: levels from it on
        are visited once per visit of the level above; prolong_scale: every prolonged correction is
        multiplied by it (1: the reference); pre_coarse / post_coarse >= 0: the smoothing counts of levels >= 1
        (-1: pre / post, the reference). All are preconditioner variants of the solver's."""
        dt = self.dtype
        arrs = [c(p, dt), c(b, dt), c(mask, dt), [c(a, dt) for a in op0]]
        assert arrs[0] is p, "p must be a contiguous array of the level dtype (updated in place)"
        n = len(self.shapes)

        def table(items):
            return (ctypes.c_void_p * n)(*[a.ctypes.data for a in items])

        P = table([arrs[0]] + self.p[1:])
        B = table([arrs[1]] + self.b[1:])
        M = table([arrs[2]] + self.m[1:])
        Dg = table([arrs[3][0]] + [o[0] for o in self.ops[1:]])
        Wx = table([arrs[3][1]] + [o[1] for o in self.ops[1:]])
        Wy = table([arrs[3][2]] + [o[2] for o in self.ops[1:]])
        Wz = table([arrs[3][3]] + [o[3] for o in self.ops[1:]])
        shapes = (ctypes.c_int * (3 * n))(*[x for s in self.shapes for x in s])
        keep = (arrs, P, B, M, Dg, Wx, Wy, Wz, shapes)  # noqa: F841 - keep buffers alive during the call
        if dt == np.float32:
            lib().orc_w_cycle_f32(P, B, M, Dg, Wx, Wy, Wz, shapes, n, F32(delta), pre, post, coarse, single_from,
                                  F32(prolong_scale), int(pre_coarse), int(post_coarse))
        else:
            lib().orc_w_cycle_f64(P, B, M, Dg, Wx, Wy, Wz, shapes, n, float(delta), pre, post, coarse, single_from,
                                  float(prolong_scale), int(pre_coarse), int(post_coarse))


def residual_norms(p, b, mask, op0, delta):
    """(sum r^2, sum b^2) in FP64 over interior fluid cells."""
    rr, bb = ctypes.c_double(0.0), ctypes.c_double(0.0)
    if p.dtype == np.float64:
        lib().orc_residual_norms_f64(c(p, np.float64), c(b, np.float64), c(mask, np.float64),
                                     *(c(a, np.float64) for a in op0), float(delta), *p.shape,
                                     ctypes.addressof(rr), ctypes.addressof(bb))
    else:
        lib().orc_residual_norms_f32(c(p), c(b), c(mask), *(c(a) for a in op0), F32(delta), *p.shape,
                                     ctypes.addressof(rr), ctypes.addressof(bb))
    return rr.value, bb.value


def relative_residual(p, b, mask, op0, delta):
    rr, bb = residual_norms(p, b, mask, op0, delta)
    return 0.0 if bb == 0.0 else float(np.sqrt(rr / bb))


def pressure_solve(u, v, w, ff, pressure, dx, dt, rho, num_vcycles, shape, levels: Levels | None = None):
    """pressure_solve.py:10-85 (reference algorithm, float32)."""
    levels = levels or Levels(shape)
    rhs = pressure_rhs(u, v, w, ff, dx, dt, rho, shape)
    op0 = build_finest_operator(ff, shape)
    p = c(pressure).copy()
    for _ in range(num_vcycles):
        levels.w_cycle(p, rhs, c(ff), op0, F32(float(dx)))
    return neumann_domain_bc(p, shape), rhs, op0


def fp64_pressure_solve(rhs, ff, shape, dx, tol=1e-12, max_cycles=200, p0=None):
    """The same W-cycle in FP64 throughout, run to ``tol``: the FP64 reference solution that GPU
    pressures are measured against."""
    levels = Levels(shape, dtype=np.float64)
    mask = c(ff, np.float64)
    op0 = build_finest_operator(mask, shape, np.float64)
    b = c(rhs, np.float64)
    p = np.zeros(shape, np.float64) if p0 is None else c(p0, np.float64).copy()
    history = []
    for _ in range(max_cycles):
        rel = relative_residual(p, b, mask, op0, dx)
        history.append(rel)
        if rel <= tol:
            break
        levels.w_cycle(p, b, mask, op0, dx)
    return p, history


def apply_operator64(p, mask, op0, delta):
    """A p in FP64 at interior fluid cells (0 elsewhere) for the finest-level operator arrays op0
    (multigrid.cl:7-43 weighted_neighbor_sum / apply_operator)."""
    d, wx, wy, wz = (np.asarray(a, np.float64) for a in op0)
    p = np.asarray(p, np.float64)
    fluid = np.zeros(p.shape, bool)
    fluid[1:-1, 1:-1, 1:-1] = np.asarray(mask)[1:-1, 1:-1, 1:-1] > 0
    ws = np.zeros_like(p)
    I = (slice(1, -1),) * 3
    ws[I] = (wx[I] * p[2:, 1:-1, 1:-1] + wx[:-2, 1:-1, 1:-1] * p[:-2, 1:-1, 1:-1]
             + wy[I] * p[1:-1, 2:, 1:-1] + wy[1:-1, :-2, 1:-1] * p[1:-1, :-2, 1:-1]
             + wz[I] * p[1:-1, 1:-1, 2:] + wz[1:-1, 1:-1, :-2] * p[1:-1, 1:-1, :-2])
    return np.where(fluid, (ws - d * p) * (1.0 / (float(delta) * float(delta))), 0.0), fluid


def fcg_solve(rhs, ff, shape, dx, p0=None, tol=1e-6, max_cycles=100, flexible=True, coarse_iterations=64,
              pre_smooth=2, post_smooth=4, single_from=0, prolong_scale=1.0, coarse_smooth=None):
    """Flexible CG (Notay, truncation 1) preconditioned by one FP32 W-cycle from zero, with the
    pressure, residual and scalars in FP64 (the product's tolerance-mode iteration; the reference
    has no counterpart). ``flexible=False`` is plain refinement p += W(r). ``coarse_iterations``:
    red-black iterations of each coarsest-level solve in the W-cycle (the reference's 64 by default);
    ``pre_smooth``/``post_smooth``: its smoothing sweeps per level (the reference's 2 and 4);
    ``single_from``: levels from it on visited once per parent visit (0: the reference's two);
    ``prolong_scale``: the factor of every prolonged correction (1: the reference's W-cycle);
    ``coarse_smooth``: (pre, post) smoothing counts of levels >= 1 (None: pre_smooth / post_smooth).
    Returns the FP64 pressure and the relative-residual history (one entry per W-cycle, the first
    for p0)."""
    levels = Levels(shape)
    ff32 = c(ff)
    op32 = build_finest_operator(ff32, shape)
    op64 = build_finest_operator(c(ff, np.float64), shape, np.float64)
    fluid = apply_operator64(np.zeros(shape), ff32, op64, dx)[1]
    b = np.where(fluid, c(rhs, np.float64), 0.0)
    x = np.zeros(shape) if p0 is None else np.where(fluid, c(p0, np.float64), 0.0)
    nb = float(np.sqrt(np.sum(b * b)))
    r = np.zeros(shape, np.float64)
    r32 = np.zeros(shape, np.float32)
    d = np.zeros(shape, np.float32)
    e = np.zeros(shape, np.float32)
    dad, rr = ctypes.c_double(0.0), ctypes.c_double(0.0)

    def update(flex):
        # orc_fcg_update: the CG scalars, direction and iterate, then r = b - A x and sum r^2 (FP64)
        lib().orc_fcg_update(e, d, x, r, r32, b, ff32, *op64, float(dx), *shape, int(flex), ctypes.addressof(dad),
                             ctypes.addressof(rr))
        return float(np.sqrt(rr.value)) / nb if nb else 0.0

    cpre, cpost = (-1, -1) if coarse_smooth is None else (int(coarse_smooth[0]), int(coarse_smooth[1]))
    hist = [update(False)]  # e = 0: only the initial residual
    while hist[-1] > tol and len(hist) <= max_cycles:
        e[...] = 0.0
        levels.w_cycle(e, r32.copy(), ff32, op32, F32(float(dx)), pre=int(pre_smooth), post=int(post_smooth),
                       coarse=int(coarse_iterations), single_from=int(single_from),
                       prolong_scale=float(prolong_scale), pre_coarse=cpre, post_coarse=cpost)
        hist.append(update(flexible))
    return x, hist


# ---- the whole step ----------------------------------------------------------------------------
class OracleSim:
    """solver.py:308-510 restated step for step on the CPU (obstacle passes always run, as in the
    reference; an empty mask makes them no-ops)."""

    def __init__(self, shape, dx, positions, velocities, obstacle=None, dt=1.0 / 240.0, flip_ratio=1.0,
                 gravity=(0.0, 0.0, -9.81), rho=1000.0, nu=1.0e-6, ppc=8, min_size=8, num_vcycles=1, tol=None,
                 coarse_iterations=64, pre_smooth=2, post_smooth=4, collider_pose=None, origin=(0.0, 0.0, 0.0),
                 prolong_scale=1.0, coarse_smooth=None):
        self.shape = tuple(int(s) for s in shape)
        self.dx, self.dt, self.flip_ratio = float(dx), float(dt), float(flip_ratio)
        self.gravity, self.rho, self.nu, self.ppc = tuple(gravity), float(rho), float(nu), ppc
        self.num_vcycles = num_vcycles
        # tol: solve each pressure to this FP64 relative residual with fcg_solve (the product's
        # tolerance mode, W-cycle preconditioner with these coarse and smoothing counts) instead of
        # the reference's fixed num_vcycles W-cycles
        self.tol = tol
        self.fcg_options = dict(coarse_iterations=coarse_iterations, pre_smooth=pre_smooth, post_smooth=post_smooth,
                                prolong_scale=prolong_scale, coarse_smooth=coarse_smooth)
        self.last_cycles = 0
        # moving colliders: collider_pose(t) -> (world triangle arrays at time t, the 9 motion parameters
        # in grid-local coordinates); each step voxelises them at the step's start time
        self.collider_pose = collider_pose
        self.origin = tuple(origin)
        self.steps_done = 0
        self.pos = c(positions).copy()
        self.vel = c(velocities).copy()
        self.obstacle = np.zeros(self.shape, np.uint8) if obstacle is None else c(obstacle, np.uint8)
        self.pressure = np.zeros(self.shape, np.float32)
        self.levels = Levels(self.shape, min_size)
        self.trace: dict[str, np.ndarray] = {}

    def step(self):
        s, dx, dt = self.shape, self.dx, self.dt
        motion = None
        if self.collider_pose is not None:
            tris, motion = self.collider_pose(self.steps_done * dt)
            mask = np.zeros(s, np.uint8)
            for t in tris:
                mask = voxelise(t, s, dx, self.origin, mask)
            self.obstacle = mask
        self.steps_done += 1
        pos_s, vel_s, u, v, w, ff, counts, offsets = particle_to_grid(self.pos, self.vel, dx, s, self.ppc)
        self.trace.update(counts=counts, offsets=offsets, sorted_pos=pos_s, sorted_vel=vel_s, p2g_u=u, p2g_v=v,
                          p2g_w=w, p2g_ff=ff)
        u, v, w, ff = grid_obstacle_bc(u, v, w, ff, self.obstacle, s, motion, dx)
        u, v, w = grid_domain_bc(u, v, w, s)
        uo, vo, wo = u, v, w
        u, v, w = update_velocity(u, v, w, ff, self.gravity, (0.0, 0.0, 0.0), self.rho, self.nu, dx, dt, s)
        u, v, w = grid_domain_bc(u, v, w, s)
        u, v, w, ff = grid_obstacle_bc(u, v, w, ff, self.obstacle, s, motion, dx)
        self.trace.update(pre_u=u, pre_v=v, pre_w=w, pressure_in=self.pressure.copy())
        if self.tol is None:
            self.pressure, rhs, op0 = pressure_solve(u, v, w, ff, self.pressure, dx, dt, self.rho, self.num_vcycles,
                                                     s, self.levels)
            self.last_cycles = self.num_vcycles
        else:
            rhs = pressure_rhs(u, v, w, ff, dx, dt, self.rho, s)
            p64, hist = fcg_solve(rhs, ff, s, dx, p0=self.pressure, tol=self.tol, **self.fcg_options)
            self.pressure = neumann_domain_bc(p64.astype(np.float32), s)
            self.last_cycles = len(hist) - 1
        self.trace.update(rhs=rhs, ff=ff, pressure=self.pressure.copy())
        u, v, w = pressure_correction(u, v, w, self.pressure, dx, dt, self.rho, s)
        u, v, w = grid_domain_bc(u, v, w, s)
        u, v, w, ff = grid_obstacle_bc(u, v, w, ff, self.obstacle, s, motion, dx)
        self.trace.update(u=u, v=v, w=w)
        vel = grid_to_particle(vel_s, pos_s, (u, v, w), (uo, vo, wo), dx, s, self.flip_ratio)
        self.trace.update(vel_g2p=vel)
        prev = pos_s.copy()
        pos = advect(pos_s, vel, dt)
        pos, vel = particle_domain_bc(pos, vel, dx, s)
        pos, vel = particle_obstacle_bc(pos, prev, vel, self.obstacle, dx, s, motion)
        self.pos, self.vel = pos, vel
        return self
