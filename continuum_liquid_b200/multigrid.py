"""Multigrid W-cycle (mirrors Solver/Kernel/multigrid.py).

Two forms are provided:

* the reference's own form: ``create_multigrid_levels`` returns per-level float32 arrays (p, b,
  mask, and the (diagonal, wx, wy, wz) operator tuple) and ``w_cycle``/``smooth``/``coarse_smooth``
  dispatch one CUDA kernel per reference kernel, with the reference's recursion;
* the packed form used by the solver: ``MultigridHierarchy`` keeps the finest operator in one byte
  per cell and the coarse operators as float4 + mask byte, builds the Galerkin coarse operators once
  per solve, and runs a whole W-cycle with one library call (capturable in a CUDA graph).

Both give the same values as the CPU restatement of the reference.
"""

from __future__ import annotations

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


def w_cycle(kernels: Backend, queue, level, p_levels, b_levels, mask_levels, operator_levels, p_level0, b_level0,
            mask_level0, operator_level0, base_delta, level_shapes, level0_shape, pre_smooth, post_smooth,
            coarse_smooth_iterations) -> None:
    """multigrid.py:53-187: one dense multigrid W-cycle for laplace(p) = b (reference layout)."""
    if level == 0:
        p, b, mask, operator, shape = p_level0, b_level0, mask_level0, operator_level0, level0_shape
    else:
        current = level - 1
        p, b, mask = p_levels[current], b_levels[current], mask_levels[current]
        operator, shape = operator_levels[current], level_shapes[current]

    if level == len(p_levels):
        coarse_smooth(kernels, queue, p, b, mask, operator, base_delta, pre_smooth + coarse_smooth_iterations, shape)
        return

    smooth(kernels, queue, p, b, mask, operator, base_delta, pre_smooth, shape)
    coarse = level
    coarse_shape = level_shapes[coarse]
    kernels.call(
        "clb_restrict_residual",
        p,
        b,
        mask,
        *operator,
        p_levels[coarse],
        b_levels[coarse],
        mask_levels[coarse],
        *operator_levels[coarse],
        float(FIELD_DTYPE(base_delta)),
        *shape,
        *coarse_shape,
        stream=queue,
    )
    args = (p_levels, b_levels, mask_levels, operator_levels, p_level0, b_level0, mask_level0, operator_level0,
            base_delta, level_shapes, level0_shape, pre_smooth, post_smooth, coarse_smooth_iterations)
    w_cycle(kernels, queue, level + 1, *args)
    w_cycle(kernels, queue, level + 1, *args)
    kernels.call("clb_prolongate", p_levels[coarse], p, mask, *coarse_shape, *shape, stream=queue)
    smooth(kernels, queue, p, b, mask, operator, base_delta, post_smooth, shape)


def smooth(kernels: Backend, queue, p, b, mask, operator, delta, iterations, shape) -> None:
    """multigrid.py:190-220: red-black Gauss-Seidel, two colour launches per iteration."""
    for _ in range(iterations):
        for parity in (0, 1):
            kernels.call("clb_rbgs_step", p, b, mask, *operator, float(FIELD_DTYPE(delta)), parity, *shape,
                         stream=queue)


def coarse_smooth(kernels: Backend, queue, p, b, mask, operator, delta, iterations, shape) -> None:
    """multigrid.py:223-249: the coarsest level smoothed in one single-block launch."""
    kernels.call("clb_coarse_smooth", p, b, mask, *operator, float(FIELD_DTYPE(delta)), int(iterations), *shape,
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
                x_from_zero: bool = False) -> None:
        """One W-cycle on level-0 unknown ``x`` and right-hand side ``rhs``. ``x_zero_outside``: the
        caller guarantees that ``x`` is 0 at every cell that is not fluid (a zeroed correction), so the
        level-0 sweeps may skip the tiles without fluid. ``x_from_zero``: the W-cycle starts from a zero
        ``x`` although ``x`` still holds a previous correction at fluid cells (it must be 0 at every
        other cell): the first sweep ignores ``x`` instead of the caller zeroing it."""
        self.struct.zero_outside = 2 if x_from_zero else (1 if x_zero_outside else 0)
        self.kernels.call_hierarchy("clb_mg_w_cycle", self.struct, x, rhs, int(pre_smooth), int(post_smooth),
                                    int(coarse_iterations), stream=queue)

    def set_sweep(self, level: int, kind: int) -> None:
        """Red-black sweep implementation of one level (see clb_mg_hierarchy.sweep); FP16 levels take
        kinds 2-6 (0 means 4)."""
        kind = int(kind)
        if kind not in (0, 1, 2, 3, 4, 5, 6):
            raise ValueError(f"unknown sweep kind {kind}")
        if self.is_fp16(level) and kind == 1:
            raise ValueError(f"level {level} is stored in FP16: sweep kinds 2-6")
        self.struct.sweep[level] = 4 if self.is_fp16(level) and kind == 0 else kind

    def sweeps(self) -> list[int]:
        return [int(self.struct.sweep[l]) for l in range(self.levels)]

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
