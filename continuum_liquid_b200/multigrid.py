"""Multigrid W-cycle (mirrors Solver/Kernel/multigrid.py).

The reference keeps five float32 arrays per level (mask, diagonal, wx, wy, wz) plus p and b, and its
host code walks the W-cycle recursion one OpenCL kernel per step. Here:

* ``MultigridHierarchy`` is the product path: the finest operator in one byte per cell, the coarse
  operators as float4 + mask byte, built once per solve, a whole W-cycle in one library call
  (capturable in a CUDA graph), fluid tiles, cluster and bottom visits;
* the reference's stage functions keep their names and arguments (``create_multigrid_levels``,
  ``w_cycle``, ``smooth``, ``coarse_smooth``) for callers that hold the reference's level arrays:
  they pack those arrays into the product formats, run the product kernels and write the coarse
  operators back where the reference's restriction leaves them.

Both give the reference's values bit for bit (tests compare them with the CPU restatement).
"""

from __future__ import annotations

import ctypes
from typing import Any

import numpy as np
import torch

from .backend import MG_MAX_LEVELS, Backend, MGHierarchy

FIELD_DTYPE = np.float32

# pressure_solve.py:61-83: W-cycle sweep counts
PRE_SMOOTH = 2
POST_SMOOTH = 4
COARSE_SMOOTH_ITERATIONS = 64


def coarse_grid_size(fine_size: int) -> int:
    """multigrid.py:12-15: coarsen cell centres while retaining one ghost cell on either side."""
    interior_size = max(0, fine_size - 2)
    return (interior_size + 1) // 2 + 2


def level_shapes_for(shape, min_size: int = 8) -> list[tuple[int, int, int]]:
    """Shapes of the levels below ``shape`` (multigrid.py:30-48 loop)."""
    shapes = []
    nx, ny, nz = (coarse_grid_size(int(s)) for s in shape)
    while nx >= min_size and ny >= min_size and nz >= min_size:
        shapes.append((nx, ny, nz))
        nx, ny, nz = coarse_grid_size(nx), coarse_grid_size(ny), coarse_grid_size(nz)
    return shapes


def create_multigrid_levels(context, shape, min_size: int = 8):
    """multigrid.py:18-50: dense float32 levels below the simulation grid (reference layout)."""
    device = context.device if isinstance(context, Backend) else torch.device(context or "cuda")
    p_levels, b_levels, mask_levels, operator_levels, level_shapes = [], [], [], [], []
    for level_shape in level_shapes_for(shape, min_size):
        alloc = lambda: torch.zeros(level_shape, dtype=torch.float32, device=device)  # noqa: E731
        p_levels.append(alloc())
        b_levels.append(alloc())
        mask_levels.append(alloc())
        operator_levels.append(tuple(alloc() for _ in range(4)))
        level_shapes.append(level_shape)
    return p_levels, b_levels, mask_levels, operator_levels, level_shapes


def _stage_cache(kernels: Backend) -> dict:
    """Per-backend workspace of the stage functions (packed hierarchies and level buffers)."""
    cache = getattr(kernels, "_stage_cache", None)
    if cache is None:
        cache = {}
        kernels._stage_cache = cache
    return cache


def stage_min_size(shape, level_shapes) -> int:
    """The ``min_size`` of ``create_multigrid_levels`` that produced ``level_shapes`` for ``shape``."""
    wanted = [tuple(int(x) for x in s) for s in level_shapes]
    for m in (8, *range(2, 65)):
        if level_shapes_for(shape, m) == wanted:
            return m
    raise ValueError(f"level shapes {wanted} are not a multigrid pyramid of {tuple(shape)}")


def _stage_hierarchy(kernels: Backend, shape, level_shapes, delta) -> "MultigridHierarchy":
    key = ("hierarchy", tuple(int(s) for s in shape), tuple(tuple(s) for s in level_shapes), float(FIELD_DTYPE(delta)))
    cache = _stage_cache(kernels)
    if key not in cache:
        cache[key] = MultigridHierarchy(kernels, shape, float(delta), stage_min_size(shape, level_shapes))
    return cache[key]


def _packed_level(kernels: Backend, shape):
    key = ("level", tuple(int(s) for s in shape))
    cache = _stage_cache(kernels)
    if key not in cache:
        cache[key] = (torch.zeros((*shape, 4), dtype=torch.float32, device=kernels.device),
                      torch.zeros(tuple(shape), dtype=torch.uint8, device=kernels.device))
    return cache[key]


def write_coarse_operators(kernels: Backend, queue, hierarchy: "MultigridHierarchy", mask_levels,
                           operator_levels) -> None:
    """The hierarchy's coarse operators into the reference's level arrays (mask as 1.0 / 0.0, then
    diagonal, wx, wy, wz): what restrict_residual (multigrid.cl:90-180) leaves there."""
    for level in range(1, hierarchy.levels):
        kernels.call("clb_mg_unpack_level", hierarchy.op[level], hierarchy.mask[level], mask_levels[level - 1],
                     *operator_levels[level - 1], *hierarchy.shapes[level], stream=queue)


def w_cycle(kernels: Backend, queue, level, p_levels, b_levels, mask_levels, operator_levels, p_level0, b_level0,
            mask_level0, operator_level0, base_delta, level_shapes, level0_shape, pre_smooth, post_smooth,
            coarse_smooth_iterations) -> None:
    """multigrid.py:53-187: one W-cycle for laplace(p) = b on the reference's level arrays.

    The finest operator (``operator_level0`` with ``mask_level0``, as build_finest_operator writes
    them) is packed into one byte per cell and the W-cycle runs on the product hierarchy; ``p_level0``
    is updated in place with the reference's values. The coarse levels' operators and masks are
    written to ``operator_levels`` / ``mask_levels`` as the reference's restriction leaves them; their
    ``p_levels`` and ``b_levels`` are the W-cycle's workspace and are not written. The reference's
    callers start a W-cycle at level 0 only (pressure_solve.py:61-83); so does this function."""
    if int(level) != 0:
        raise ValueError("w_cycle runs whole W-cycles from level 0 (the level argument of the reference's "
                         "recursion); coarse levels are visited inside it")
    h = _stage_hierarchy(kernels, level0_shape, level_shapes, base_delta)
    invalid = torch.zeros(1, dtype=torch.int32, device=kernels.device)
    kernels.call("clb_mg_pack_finest", mask_level0, *operator_level0, h.op0, invalid, *level0_shape, stream=queue)
    if int(invalid.item()):
        raise ValueError(f"operator_level0 is not a finest-level operator at {int(invalid.item())} cells "
                         "(diagonal 0..7 and 0/1 weights, as build_finest_operator writes them)")
    h.build_coarse(queue=queue)
    h.w_cycle(p_level0, b_level0, pre_smooth, post_smooth, coarse_smooth_iterations, queue=queue)
    write_coarse_operators(kernels, queue, h, mask_levels, operator_levels)


def smooth(kernels: Backend, queue, p, b, mask, operator, delta, iterations, shape) -> None:
    """multigrid.py:190-220: red-black Gauss-Seidel on one level of the reference's arrays (packed
    into the product's coarse-level format for the product sweep kernel)."""
    op4, mask8 = _packed_level(kernels, shape)
    kernels.call("clb_mg_pack_level", mask, *operator, op4, mask8, *shape, stream=queue)
    kernels.call("clb_mg_smooth_level", p, b, op4, mask8, float(FIELD_DTYPE(delta)), int(iterations), *shape,
                 stream=queue)


def coarse_smooth(kernels: Backend, queue, p, b, mask, operator, delta, iterations, shape) -> None:
    """multigrid.py:223-249: the coarsest level smoothed in one single-block launch (the product's
    coarse solve on the packed level)."""
    op4, mask8 = _packed_level(kernels, shape)
    kernels.call("clb_mg_pack_level", mask, *operator, op4, mask8, *shape, stream=queue)
    kernels.call("clb_mg_coarse_solve_level", p, b, op4, mask8, float(FIELD_DTYPE(delta)), int(iterations), *shape,
                 stream=queue)


class MultigridHierarchy:
    """Packed level pyramid for the product solve path (clb_mg_hierarchy).

    Level 0 is the simulation grid: its operator (``op0``, uint8 per cell) is written by
    ``rhs_operator`` each step. Coarse levels own p, b (float32), mask (uint8) and op (float4 as a
    float32 [..., 4] tensor). ``shapes[l]`` includes the ghost layer, as in the reference.

    ``fp16_max_size`` > 0 stores every coarse level whose largest extent is at most that size in FP16
    (p, b and op as float16, scaled as described in csrc/mg_half.cuh; no counterpart in the
    reference), provided at least the two coarsest levels qualify. A W-cycle then needs
    ``norms[0]`` to hold the squared norm of its right-hand side (the residual kernels leave it
    there), and those levels use the per-cell or the fused sweep kinds (not the row-vector kind 1).
    """

    def __init__(self, kernels: Backend, grid_shape, dx: float, min_size: int = 8, fused_min_cells: int = 20**3,
                 fp16_max_size: int = 0, fluid_tiles: bool = True):
        self.kernels = kernels
        self.grid_shape = tuple(int(s) for s in grid_shape)
        self.dx = float(dx)
        self.shapes = [self.grid_shape, *level_shapes_for(self.grid_shape, min_size)]
        if len(self.shapes) > MG_MAX_LEVELS:
            raise ValueError(f"{len(self.shapes)} multigrid levels exceed the limit of {MG_MAX_LEVELS}")
        device = kernels.device
        levels = len(self.shapes)
        self.fp16_level = 0
        if fp16_max_size > 0:
            first = next((l for l in range(1, levels) if max(self.shapes[l]) <= fp16_max_size), 0)
            if 1 <= first <= levels - 2:
                self.fp16_level = first
        self.op0 = torch.zeros(self.grid_shape, dtype=torch.uint8, device=device)
        self.p: list[torch.Tensor | None] = [None]
        self.b: list[torch.Tensor | None] = [None]
        self.mask: list[torch.Tensor | None] = [None]
        self.op: list[torch.Tensor | None] = [None]
        for l, shape in enumerate(self.shapes[1:], start=1):
            dt = torch.float16 if self.is_fp16(l) else torch.float32
            self.p.append(torch.zeros(shape, dtype=dt, device=device))
            self.b.append(torch.zeros(shape, dtype=dt, device=device))
            self.mask.append(torch.zeros(shape, dtype=torch.uint8, device=device))
            self.op.append(torch.zeros((*shape, 4), dtype=dt, device=device))
        self.fp16_scale = torch.zeros(4, dtype=torch.float32, device=device)
        self.fp16_inexact = torch.zeros(1, dtype=torch.int32, device=device)
        self.struct = MGHierarchy()
        self.struct.levels = len(self.shapes)
        for l, shape in enumerate(self.shapes):
            for a in range(3):
                self.struct.shape[l][a] = shape[a]
        # multigrid.py:65 base_delta is passed as FIELD_DTYPE(base_delta) to every level
        self.struct.delta = float(FIELD_DTYPE(self.dx))
        self.struct.op0 = self.op0.data_ptr()
        for l in range(1, len(self.shapes)):
            self.struct.p[l] = self.p[l].data_ptr()
            self.struct.b[l] = self.b[l].data_ptr()
            self.struct.mask[l] = self.mask[l].data_ptr()
            self.struct.op[l] = self.op[l].data_ptr()
        # second buffers for the fused red-black iteration on every level of at least fused_min_cells
        # cells (smaller levels are served by the single-block bottom visit or two-launch sweeps)
        self.alt: list[torch.Tensor | None] = []
        for l, shape in enumerate(self.shapes):
            big = int(np.prod(shape)) >= fused_min_cells
            dt = torch.float16 if self.is_fp16(l) else torch.float32
            self.alt.append(torch.zeros(shape, dtype=dt, device=device) if big else None)
            if big:
                self.struct.alt[l] = self.alt[l].data_ptr()
        self.tuning: dict | None = None  # per-level sweep timings from the autotuner (ms per iteration)
        cells = int(np.prod(self.grid_shape))
        self.partials = torch.zeros((kernels.residual_partials(cells), 2), dtype=torch.float64, device=device)
        self.norms = torch.zeros(2, dtype=torch.float64, device=device)
        self.struct.fp16_level = self.fp16_level
        self.struct.fp16_scale = self.fp16_scale.data_ptr()
        self.struct.rhs_norms = self.norms.data_ptr()
        self.struct.fp16_inexact = self.fp16_inexact.data_ptr()
        # fluid tiles per level (csrc/mg_tiles.cuh): inside a W-cycle the FP32 levels' sweeps,
        # restrictions and prolongations visit only the tiles that hold fluid
        self.tiles: list[torch.Tensor] = []
        self.tile_counts = torch.zeros(MG_MAX_LEVELS, dtype=torch.int32, device=device)
        if fluid_tiles:
            for l, shape in enumerate(self.shapes):
                cap = int(kernels.lib.clb_mg_tile_capacity(*shape, 1 if l == 0 else 0))
                self.tiles.append(torch.zeros(max(cap, 1), dtype=torch.int32, device=device))
                self.struct.tiles[l] = self.tiles[l].data_ptr()
            self.struct.tile_counts = self.tile_counts.data_ptr()
            # 3-D fluid tiles of level 0 for the fused level-0 visit (sweep kind 7, csrc/mg_level0.cuh)
            cap = int(kernels.lib.clb_mg_fused_tile_capacity(*self.grid_shape))
            self.fused_tiles = torch.zeros(max(cap, 1), dtype=torch.int32, device=device)
            self.fused_tile_count = torch.zeros(1, dtype=torch.int32, device=device)
            self.struct.fused_tiles = self.fused_tiles.data_ptr()
            self.struct.fused_tile_count = self.fused_tile_count.data_ptr()
        # the fluid cells of the three coarsest levels for the one-launch visits of the third-coarsest
        # level (csrc/mg_cluster.cuh), listed once per solve by build_coarse
        cap = int(kernels.lib.clb_mg_cluster_list_capacity(ctypes.byref(self.struct)))
        self.cluster_lists = torch.zeros(max(cap, 1), dtype=torch.int32, device=device) if cap > 0 else None
        if self.cluster_lists is not None:
            self.struct.cluster_lists = self.cluster_lists.data_ptr()
        for l in range(1, levels):
            if self.is_fp16(l):
                self.struct.sweep[l] = 4

    def is_fp16(self, level: int) -> bool:
        return self.fp16_level > 0 and level >= self.fp16_level

    def fp16_inexact_entries(self) -> int:
        """Operator entries of the FP16 levels that FP16 does not hold exactly (last build_coarse)."""
        return int(self.fp16_inexact.item()) if self.fp16_level else 0

    @property
    def levels(self) -> int:
        return len(self.shapes)

    def rhs_operator(self, velocity, fluid_fraction, rhs, dt: float, rho: float, queue=None) -> None:
        """pressure_rhs + build_finest_operator (pressure_solve.py:35-59) into rhs and op0."""
        u, v, w = velocity
        self.kernels.call("clb_mg_rhs_operator", u, v, w, fluid_fraction, rhs, self.op0,
                          float(FIELD_DTYPE(float(rho) / float(dt))), float(FIELD_DTYPE(1.0 / self.dx)), *self.grid_shape,
                          stream=queue)

    def build_coarse(self, queue=None) -> None:
        """Galerkin coarse operators of every level (operator part of multigrid.cl:90-180)."""
        self.kernels.call_hierarchy("clb_mg_build_coarse", self.struct, stream=queue)

    def w_cycle(self, x, rhs, pre_smooth=PRE_SMOOTH, post_smooth=POST_SMOOTH,
                coarse_iterations=COARSE_SMOOTH_ITERATIONS, queue=None, x_zero_outside: bool = False,
                x_from_zero: bool = False, prolong_scale: float = 1.0, coarse_smooth=None) -> None:
        """One W-cycle on level-0 unknown ``x`` and right-hand side ``rhs``. ``x_zero_outside``: the
        caller guarantees that ``x`` is 0 at every cell that is not fluid (a zeroed correction), so the
        level-0 sweeps may skip the tiles without fluid. ``x_from_zero``: the W-cycle starts from a zero
        ``x`` although ``x`` still holds a previous correction at fluid cells (it must be 0 at every
        other cell): the first sweep ignores ``x`` instead of the caller zeroing it.
        ``prolong_scale``: every prolonged correction is multiplied by it (1: the reference's W-cycle;
        no counterpart in the reference, see clb_mg_hierarchy.prolong_scale). ``coarse_smooth``: (pre, post)
        smoothing counts of levels >= 1 (None: ``pre_smooth`` / ``post_smooth`` on every level, the
        reference)."""
        self.struct.zero_outside = 2 if x_from_zero else (1 if x_zero_outside else 0)
        self.struct.prolong_scale = float(prolong_scale)
        self.set_coarse_smooth(coarse_smooth)
        self.kernels.call_hierarchy("clb_mg_w_cycle", self.struct, x, rhs, int(pre_smooth), int(post_smooth),
                                    int(coarse_iterations), stream=queue)

    def set_coarse_smooth(self, coarse_smooth) -> None:
        """Smoothing counts (pre, post) of levels >= 1 for the W-cycles that follow (None: the W-cycle's)."""
        if coarse_smooth is None:
            self.struct.coarse_smoothing = 0
            return
        pre, post = (int(x) for x in coarse_smooth)
        if pre < 0 or post < 0:
            raise ValueError("coarse_smooth counts must be >= 0")
        self.struct.coarse_smoothing = 1
        self.struct.coarse_pre_smooth, self.struct.coarse_post_smooth = pre, post

    def set_sweep(self, level: int, kind: int) -> None:
        """Red-black sweep implementation of one level (see clb_mg_hierarchy.sweep); FP16 levels take
        kinds 2-6 (0 means 4); kind 7 on level 0 runs the W-cycle's level-0 visit as fused tile launches
        (tolerance-mode W-cycles from a zero correction)."""
        kind = int(kind)
        if kind not in (0, 1, 2, 3, 4, 5, 6, 7):
            raise ValueError(f"unknown sweep kind {kind}")
        if kind == 7 and level != 0:
            raise ValueError("sweep kind 7 (the fused level-0 visit) is for level 0 only")
        if self.is_fp16(level) and kind == 1:
            raise ValueError(f"level {level} is stored in FP16: sweep kinds 2-6")
        self.struct.sweep[level] = 4 if self.is_fp16(level) and kind == 0 else kind

    def sweeps(self) -> list[int]:
        return [int(self.struct.sweep[l]) for l in range(self.levels)]

    def level0_iteration(self, x_in, x_out, rhs, mode: int, queue=None) -> None:
        """One launch of the fused level-0 kernel (clb_mg_level0_iteration): mode 1 = from zero, 2 = with
        the restriction into level 1, 3 = both, 4 = with the prolongation of level 1's p, 0 = neither."""
        self.kernels.call_hierarchy("clb_mg_level0_iteration", self.struct, x_in, x_out, rhs, int(mode),
                                    stream=queue)

    def fused_tile_cells(self) -> int:
        """Grid cells covered by the listed fused level-0 tiles (after build_coarse)."""
        n = int(self.fused_tile_count.item())
        if n == 0:
            return 0
        nx, ny, nz = self.grid_shape
        tj, tk = -(-(ny - 2) // 8), -(-(nz - 2) // 32)
        t = self.fused_tiles[:n].cpu().numpy().astype(np.int64)
        a, b, c = t // (tj * tk), (t // tk) % tj, t % tk
        ext = lambda start, size, n_: np.minimum(start + size, n_) - start
        return int(np.sum(ext(1 + 8 * a, 8, nx) * ext(1 + 8 * b, 8, ny) * ext(1 + 32 * c, 32, nz)))

    def smooth(self, level: int, iterations: int, x=None, rhs=None, queue=None, zero_outside: bool = False) -> None:
        """``iterations`` red-black Gauss-Seidel iterations on one level. ``zero_outside``: the caller
        guarantees that the level's p (``x`` on level 0) is 0 at every cell that is not fluid, so an
        FP32 level is swept on its fluid tiles only (the values are the same)."""
        self.struct.zero_outside = 1 if zero_outside else 0
        self.kernels.call_hierarchy("clb_mg_smooth", self.struct, int(level), x, rhs, int(iterations), stream=queue)

    def residual_norms(self, p, rhs, r_out=None, queue=None) -> torch.Tensor:
        """Device tensor [sum r^2, sum b^2] (FP64) over interior fluid cells of level 0."""
        is_double = 1 if p.dtype == torch.float64 else 0
        self.kernels.call("clb_mg_residual_norms", p, is_double, rhs, self.op0, float(FIELD_DTYPE(self.dx)),
                          *self.grid_shape, r_out, self.partials, self.norms, stream=queue)
        return self.norms

    def level_arrays(self, level: int) -> dict[str, Any]:
        """Host copies of one level (tests and diagnostics)."""
        if level == 0:
            return {"op0": self.op0.cpu().numpy()}
        return {  # FP16 levels are returned as float32 (their p and b in scaled units)
            "p": self.p[level].float().cpu().numpy(),
            "b": self.b[level].float().cpu().numpy(),
            "mask": self.mask[level].cpu().numpy(),
            "op": self.op[level].float().cpu().numpy(),
        }


def unpack_op0(op0: np.ndarray) -> tuple[np.ndarray, ...]:
    """Decode a packed level-0 operator into the reference's float arrays
    (mask>0 flag, diagonal, wx, wy, wz)."""
    o = op0.astype(np.uint32)
    return (
        ((o >> 6) & 1).astype(np.float32),
        (o & 7).astype(np.float32),
        ((o >> 3) & 1).astype(np.float32),
        ((o >> 4) & 1).astype(np.float32),
        ((o >> 5) & 1).astype(np.float32),
    )


__all__ = [
    "coarse_grid_size",
    "level_shapes_for",
    "create_multigrid_levels",
    "w_cycle",
    "smooth",
    "coarse_smooth",
    "MultigridHierarchy",
    "unpack_op0",
]
