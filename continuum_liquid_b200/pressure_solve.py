"""Pressure solve and projection (mirrors Solver/Kernel/pressure_solve.py).

``pressure_solve`` keeps the reference's signature and algorithm (pressure_rhs,
build_finest_operator, ``num_vcycles`` W-cycles, Neumann ghost copy) and runs it through
``PressureSolver``, writing the reference's outputs (``rhs``, the finest operator arrays and the coarse
operators) into the caller's arrays.

``PressureSolver`` is the product path behind the same stage: the packed multigrid hierarchy plus

* parity mode (``tol=None``): exactly ``num_vcycles`` W-cycles on the pressure, as the reference;
* tolerance mode (``tol=1e-6``): mixed-precision iterative refinement. The pressure is accumulated
  in FP64; each refinement computes the FP64 residual r = b - A p (and its norm), solves A e = r
  with one FP32 W-cycle from e = 0 and adds e to p, until ||r||_2 / ||b||_2 <= tol over the
  interior fluid cells. A W-cycle is an affine map, so ``method="refine"`` is the same iteration
  as running W-cycles on p, with the rounding of the FP32 residual (which cannot reach 1e-6 by
  itself) removed. ``method="fcg"`` (the default) applies the same W-cycle corrections along
  flexible conjugate-gradient directions (Notay's FCG with truncation 1), which needs fewer
  W-cycles for the same tolerance; the accumulation, residual and norms stay FP64.

The solution of a tolerance-mode solve is the FP64 pressure (``pressure64``): its float32
rounding, written to ``pressure``, cannot hold a relative residual of 1e-6 on fine grids, so the
projection uses the FP64 pressure when one exists.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import boundary_conditions, multigrid
from .backend import Backend

FIELD_DTYPE = np.float32


def pressure_solve(kernels: Backend, multigrid_kernels, boundary_kernels, queue, velocity, fluid_fraction, pressure,
                   rhs, p_levels, b_levels, mask_levels, operator_level0, operator_levels, multigrid_level_shapes, dx,
                   dt, rho, num_vcycles, grid_shape):
    """pressure_solve.py:10-85: right-hand side, finest operator, ``num_vcycles`` W-cycles on the
    previous pressure and the Neumann ghost copy, by the product solver (the packed hierarchy, its
    W-cycle bit for bit the reference's). ``rhs`` and ``operator_level0`` receive what the reference's
    pressure_rhs and build_finest_operator write, ``operator_levels`` / ``mask_levels`` the coarse
    operators; ``p_levels`` and ``b_levels`` are workspace and are not written."""
    key = ("solver", tuple(int(s) for s in grid_shape), tuple(tuple(s) for s in multigrid_level_shapes),
           float(FIELD_DTYPE(dx)))
    cache = multigrid._stage_cache(kernels)
    if key not in cache:
        cache[key] = PressureSolver(kernels, grid_shape, float(dx),
                                    min_size=multigrid.stage_min_size(grid_shape, multigrid_level_shapes))
    ps = cache[key]
    stream = queue if queue is not None else torch.cuda.current_stream(kernels.device)
    with torch.cuda.stream(stream):
        ps.solve(velocity, fluid_fraction, pressure, dt, rho, num_vcycles=int(num_vcycles), tol=None)
        rhs.copy_(ps.rhs)
        kernels.call("clb_mg_unpack_finest", ps.hierarchy.op0, *operator_level0, *grid_shape)
        multigrid.write_coarse_operators(kernels, None, ps.hierarchy, mask_levels, operator_levels)
    return pressure


def pressure_correction(kernels: Backend, queue, velocity, pressure, dx, dt, rho, grid_shape):
    """pressure_solve.py:88-114."""
    nx, ny, nz = grid_shape
    u, v, w = velocity
    kernels.call("clb_pressure_correction", u, v, w, pressure, float(FIELD_DTYPE(float(dt) / float(rho))),
                 float(FIELD_DTYPE(1.0 / float(dx))), nx, ny, nz, stream=queue)
    return velocity


@dataclass
class SolveStats:
    """Per-solve record (added to the reference's stats messages): W-cycles run, final relative
    residual (FP64, None in parity mode unless measured) and wall time of the solve in ms."""

    cycles: int = 0
    rel_residual: float | None = None
    initial_rel_residual: float | None = None
    ms: float = 0.0
    history: list = field(default_factory=list)
    events: tuple | None = None  # CUDA events bracketing the solve on its stream
    warm_start: str = "previous"  # initial guess used: "previous" step's pressure or "learned"
    learned_rel_residual: float | None = None  # relative residual of the network's guess, when tried

    def device_ms(self) -> float:
        """Device time of the solve from its CUDA events (synchronises on the end event)."""
        if self.events is None:
            return self.ms
        self.events[1].synchronize()
        return self.events[0].elapsed_time(self.events[1])


# The tolerance mode's W-cycle preconditioner settings the benchmark chooses at 256^3 (no counterpart
# in the reference, whose fixed-cycle W-cycle keeps its 2 / 4 / 64 counts and unscaled prolongation):
# pass them to PressureSolver, StepOptions or BatchedFlip, e.g. StepOptions(tol=1e-6, **TUNED_PRECONDITIONER)
TUNED_PRECONDITIONER = {"coarse_iterations": 0, "pre_smooth": 1, "post_smooth": 2, "prolong_scale": 1.8,
                        "coarse_smooth": (1, 0)}

METHODS = ("fcg", "refine")


def ptr_of(t: torch.Tensor) -> int:
    return t.data_ptr()


class PressureSolver:
    """Packed-layout pressure solve for one grid (allocates its workspace once).

    In tolerance mode one refinement is: e = 0; one W-cycle on A e = r; then either
    p64 <- p64 + e (``refine``, clb_mg_ir_step) or the flexible-CG update along d = e + beta d
    (``fcg``, clb_mg_fcg_dots + clb_mg_fcg_step), each fused with the FP64 residual r = b - A p64
    and its norms. The FP64 pressure (and the FCG direction) alternate between two buffers, so two
    CUDA graphs (one per direction) capture the refinement. The host reads the residual norm only
    when the refinement count predicted from the observed contraction rate has run, so most
    refinements are replayed back to back without a host round trip.
    """

    def __init__(self, kernels: Backend, grid_shape, dx: float, min_size: int = 8, max_cycles: int = 100,
                 autotune: bool = True, method: str = "fcg", coarse_fp16: bool = False, fp16_max_size: int = 64,
                 coarse_iterations: int = multigrid.COARSE_SMOOTH_ITERATIONS,
                 pre_smooth: int = multigrid.PRE_SMOOTH, post_smooth: int = multigrid.POST_SMOOTH,
                 fused_level0: bool = False, device_loop: bool = False, prolong_scale: float = 1.0,
                 coarse_smooth=None):
        if method not in METHODS:
            raise ValueError(f"unknown pressure solve method {method!r} (expected one of {METHODS})")
        self.coarse_fp16 = bool(coarse_fp16)
        self.kernels = kernels
        self.grid_shape = tuple(int(s) for s in grid_shape)
        self.dx = float(dx)
        self.max_cycles = int(max_cycles)
        self.method = method
        # red-black iterations (beyond pre-smoothing) of each coarsest-level solve inside the tolerance
        # mode's W-cycle; the reference's 64 by default (fixed-cycle mode always uses 64)
        self.coarse_iterations = int(coarse_iterations)
        if self.coarse_iterations < 0:
            raise ValueError("coarse_iterations must be >= 0")
        # red-black iterations before and after the coarse-grid correction on every level of the
        # tolerance mode's W-cycle preconditioner; the reference's 2 and 4 by default (fixed-cycle mode
        # always uses those)
        self.pre_smooth, self.post_smooth = int(pre_smooth), int(post_smooth)
        # factor of every correction the tolerance mode's W-cycle prolongs (no counterpart in the
        # reference, whose piecewise-constant prolongation is 1; fixed-cycle mode always uses 1). About
        # 1.7 over-corrects what the constant prolongation under-corrects: at 256^3 the flexible CG then
        # needs 8 instead of 13 cycles per solve
        self.prolong_scale = float(prolong_scale)
        if not self.prolong_scale > 0.0:
            raise ValueError("prolong_scale must be > 0")
        # smoothing counts (pre, post) of levels >= 1 in the tolerance mode's W-cycle (None: pre_smooth and
        # post_smooth on every level, as the reference). With the scaled prolongation the coarse levels'
        # post-smoothing can go: (1, 0) needs 0-1 more cycles and each cycle is ~20 % cheaper at 256^3
        self.coarse_smooth = None if coarse_smooth is None else tuple(int(x) for x in coarse_smooth)
        if self.coarse_smooth is not None and (len(self.coarse_smooth) != 2 or min(self.coarse_smooth) < 0):
            raise ValueError("coarse_smooth must be a pair of counts >= 0")
        # fused_level0: the tolerance mode's W-cycles run level 0 as fused tile launches (sweep kind 7,
        # csrc/mg_level0.cuh), with the values of the launch-per-step path. Off by default: at 256^3 the
        # recomputed halo costs more instructions than the four launches it saves
        self.fused_level0 = bool(fused_level0)
        # device_loop: with CUDA graphs, tolerance-mode solves after the first run as one graph that
        # loops on the device until the tolerance (clb_solve_loop_*, a WHILE conditional node): no host
        # round trip between refinements. Off by default: at 256^3 it is as fast as the host loop (the
        # loop's device-side body launches cost what the host's few residual reads did), and a profiler
        # sees no kernel inside it
        self.device_loop = bool(device_loop)
        self._loop = None  # ctypes handle of the loop graph
        self._loop_key = None
        if self.pre_smooth < 0 or self.post_smooth < 0 or self.pre_smooth + self.post_smooth == 0:
            raise ValueError("pre_smooth and post_smooth must be >= 0 and not both 0")
        # FP16 storage of the coarse levels of at most fp16_max_size cells per side (tolerance mode only:
        # the W-cycle then reads the squared norm of its right-hand side from the residual kernels)
        self.hierarchy = multigrid.MultigridHierarchy(kernels, self.grid_shape, dx, min_size,
                                                      fp16_max_size=fp16_max_size if coarse_fp16 else 0)
        device = kernels.device
        self.cells = int(np.prod(self.grid_shape))
        self.rhs = torch.zeros(self.grid_shape, dtype=torch.float32, device=device)
        self.residual = torch.zeros(self.grid_shape, dtype=torch.float32, device=device)
        self.correction = torch.zeros(self.grid_shape, dtype=torch.float32, device=device)
        self.p64 = [torch.zeros(self.grid_shape, dtype=torch.float64, device=device) for _ in range(2)]
        self.cur = 0  # index of the FP64 buffer holding the current pressure
        # flexible-CG direction (ping-pong like p64), scalars {alpha, beta, d.Ad, has_direction} and
        # the partial sums of its dot products (4 doubles per block)
        self.direction = [torch.zeros(self.grid_shape, dtype=torch.float32, device=device) for _ in range(2)]
        self.fcg_state = torch.zeros(4, dtype=torch.float64, device=device)
        blocks = kernels.residual_partials(self.cells)
        self.fcg_partials = torch.zeros(4 * blocks, dtype=torch.float64, device=device)
        self.solved64 = False  # whether pressure64 holds the last solve's FP64 pressure
        self.norms_host = torch.zeros(2, dtype=torch.float64, pin_memory=True)
        self._graphs: list[torch.cuda.CUDAGraph | None] = [None, None]
        self.autotune = autotune
        self.tuned = False
        self.graph_replays = 0  # refinements replayed from graphs so far (host-loop graphs and the device loop)
        self.graph_launches = 0  # kernels inside one refinement graph
        self.host_batch = 8  # most refinements the host loop runs between two reads of the residual
        self.loop_refinements = 0  # refinements run by the device loop (each also runs one check kernel)
        self.loop_cycles = torch.zeros(1, dtype=torch.int32, device=device)
        self.loop_history = torch.zeros(self.max_cycles + 2, dtype=torch.float64, device=device)
        self._loop_host = torch.zeros(self.max_cycles + 3, dtype=torch.float64, pin_memory=True)

    # -- pieces ---------------------------------------------------------------------------------
    def prepare(self, velocity, fluid_fraction, dt, rho, queue=None) -> None:
        """Right-hand side, packed finest operator and the Galerkin coarse operators."""
        self.hierarchy.rhs_operator(velocity, fluid_fraction, self.rhs, dt, rho, queue=queue)
        self.hierarchy.build_coarse(queue=queue)

    def _relative(self, norms: torch.Tensor) -> float:
        self.norms_host.copy_(norms, non_blocking=True)
        torch.cuda.current_stream(self.kernels.device).synchronize()
        rr, bb = float(self.norms_host[0]), float(self.norms_host[1])
        return 0.0 if bb == 0.0 else math.sqrt(rr / bb)

    def relative_residual(self, pressure, queue=None) -> float:
        """FP64 ||b - A p|| / ||b|| of a float32 or float64 pressure against the prepared system."""
        return self._relative(self.hierarchy.residual_norms(pressure, self.rhs, queue=queue))

    @property
    def pressure64(self) -> torch.Tensor:
        """The FP64 pressure of the last tolerance-mode solve (0 off the interior fluid)."""
        return self.p64[self.cur]

    def refine_once(self, src: int, queue=None) -> None:
        """One refinement from FP64 buffer ``src`` into the other one."""
        h = self.hierarchy
        # the correction starts from 0: its buffer is 0 outside the fluid (zeroed once per solve, and
        # the W-cycle writes 0 to every cell that is not fluid), so the W-cycle's first sweep ignores
        # the previous correction at fluid cells instead of a fill of the whole buffer
        kind0 = int(h.struct.sweep[0])
        if self.fused_level0:
            h.struct.sweep[0] = 7
        try:
            h.w_cycle(self.correction, self.residual, pre_smooth=self.pre_smooth, post_smooth=self.post_smooth,
                      coarse_iterations=self.coarse_iterations, queue=queue, x_from_zero=True,
                      prolong_scale=self.prolong_scale, coarse_smooth=self.coarse_smooth)
        finally:
            h.struct.sweep[0] = kind0
        delta = float(FIELD_DTYPE(self.dx))
        if self.method == "fcg":
            self.kernels.call("clb_mg_fcg_dots", self.correction, self.direction[src], self.residual, h.op0, delta,
                              *self.grid_shape, self.fcg_partials, self.fcg_state, stream=queue)
            self.kernels.call("clb_mg_fcg_step", self.p64[src], self.correction, self.direction[src],
                              self.p64[1 - src], self.direction[1 - src], self.fcg_state, self.rhs, h.op0, delta,
                              *self.grid_shape, self.residual, h.partials, h.norms, stream=queue)
        else:
            self.kernels.call("clb_mg_ir_step", self.p64[src], self.correction, self.p64[1 - src], self.rhs, h.op0,
                              delta, *self.grid_shape, self.residual, h.partials, h.norms, stream=queue)

    def _refine(self, use_graph: bool) -> None:
        src = self.cur
        if not use_graph:
            self.refine_once(src)
        elif self._graphs[src] is None:
            # the first refinement in this direction runs eagerly on a side stream (warming up the
            # launches), then is captured without being replayed
            stream = torch.cuda.current_stream(self.kernels.device)
            side = torch.cuda.Stream(self.kernels.device)
            side.wait_stream(stream)
            with torch.cuda.stream(side):
                self.refine_once(src)
            stream.wait_stream(side)
            graph = torch.cuda.CUDAGraph()
            before = self.kernels.launch_count()
            with torch.cuda.graph(graph):
                self.refine_once(src)
            self.graph_launches = self.kernels.launch_count() - before
            self._graphs[src] = graph
        else:
            self._graphs[src].replay()
            self.graph_replays += 1
        self.cur = 1 - src

    # -- solves ---------------------------------------------------------------------------------
    def solve(self, velocity, fluid_fraction, pressure, dt, rho, num_vcycles: int = 1, tol: float | None = None,
              use_graph: bool = True, measure: bool = False, warm_start=None, solid=None) -> SolveStats:
        """Solve for ``pressure`` in place (warm-started from its current contents) and apply the
        Neumann ghost copy. ``tol=None`` runs ``num_vcycles`` W-cycles (reference semantics).

        ``warm_start`` (tolerance mode): a callable (rhs, op0, solid, p_prev) -> candidate pressure or
        None; the candidate replaces the previous-step pressure as the initial guess only when its
        FP64 relative residual is lower."""
        stats = SolveStats()
        t0 = time.perf_counter()
        stats.events = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        stats.events[0].record()
        self.prepare(velocity, fluid_fraction, dt, rho)
        h = self.hierarchy
        if self.autotune and not self.tuned:
            # sweep kinds are chosen on the first real operator, before any graph captures them
            from .autotune import tune_hierarchy

            tune_hierarchy(h, self.correction, self.residual)
            self.tuned = True
        if tol is None:
            if h.fp16_level:
                raise ValueError("FP16 coarse levels are a tolerance-mode option (tol=...)")
            self.solved64 = False
            for _ in range(int(num_vcycles)):
                h.w_cycle(pressure, self.rhs)
            stats.cycles = int(num_vcycles)
            if measure:
                stats.rel_residual = self.relative_residual(pressure)
        else:
            self.solve_prepared(pressure, tol, use_graph=use_graph, warm_start=warm_start, solid=solid, stats=stats)
        boundary_conditions.neumann_domain_bc(self.kernels, None, pressure, self.grid_shape)
        stats.events[1].record()
        stats.ms = (time.perf_counter() - t0) * 1e3
        return stats

    def solve_prepared(self, pressure, tol: float, use_graph: bool = True, warm_start=None, solid=None,
                       stats: SolveStats | None = None) -> SolveStats:
        """The tolerance-mode iteration on the system already in ``rhs`` and the hierarchy (after
        ``prepare``), from the initial guess ``pressure`` (float32, updated with the result)."""
        stats = stats or SolveStats()
        h = self.hierarchy
        self.cur = 0
        if self.method == "fcg":
            self.direction[0].zero_()
            self.direction[1].zero_()
            self.fcg_state.zero_()
        # the step kernels skip cells outside the fluid: both FP64 buffers start at 0 there; so does
        # the correction (the fluid of the last solve may have moved)
        self.p64[1].zero_()
        self.correction.zero_()
        self.kernels.call("clb_mg_ir_init", pressure, h.op0, self.p64[0], *self.grid_shape)
        rel = self._relative(h.residual_norms(self.p64[0], self.rhs, r_out=self.residual))
        if warm_start is not None:
            guess = warm_start(self.rhs, h.op0, solid, pressure)
            if guess is not None:
                rel_net = self.relative_residual(guess)
                stats.learned_rel_residual = rel_net
                if rel_net < rel:
                    self.kernels.call("clb_mg_ir_init", guess, h.op0, self.p64[0], *self.grid_shape)
                    rel = self._relative(h.residual_norms(self.p64[0], self.rhs, r_out=self.residual))
                    stats.warm_start = "learned"
        stats.initial_rel_residual = rel
        stats.history.append(rel)
        if use_graph and self.device_loop and self._loop is not None and self._loop_key == self._key(tol):
            if rel > tol:
                rel = self._run_loop(stats)
            stats.rel_residual = rel
            return self._finish(pressure, stats)
        rate = None
        while rel > tol and stats.cycles < self.max_cycles:
            # refinements to run before the next host check: one less than predicted, at least 1
            batch = 1
            if rate is not None and 0.0 < rate < 1.0:
                batch = max(1, int(math.ceil(math.log(tol / rel) / math.log(rate))) - 1)
            batch = min(batch, self.max_cycles - stats.cycles, self.host_batch)
            for _ in range(batch):
                self._refine(use_graph)
            previous = rel
            stats.cycles += batch
            rel = self._relative(h.norms)
            stats.history.append(rel)
            rate = (rel / previous) ** (1.0 / batch) if previous > 0 and stats.cycles > 1 else None
        stats.rel_residual = rel
        if use_graph and self.device_loop and self._loop_key != self._key(tol):
            self._build_loop(tol)  # later solves loop on the device (the launches are warm now)
        return self._finish(pressure, stats)

    def _finish(self, pressure, stats: SolveStats) -> SolveStats:
        self.kernels.call("clb_mg_ir_store", self.p64[self.cur], pressure, self.cells)
        self.kernels.call("clb_neumann_domain_bc_f64", self.p64[self.cur], *self.grid_shape)
        self.solved64 = True
        return stats

    # -- the device loop ------------------------------------------------------------------------
    def _key(self, tol: float):
        return (float(tol), self.max_cycles, self.method, self.pre_smooth, self.post_smooth, self.coarse_iterations,
                self.fused_level0)

    def _build_loop(self, tol: float) -> None:
        import ctypes

        self.release_loop()
        h = self.hierarchy
        kind0 = int(h.struct.sweep[0])
        if self.fused_level0:
            h.struct.sweep[0] = 7
        h.struct.prolong_scale = self.prolong_scale  # read when the loop's refinement is captured
        h.set_coarse_smooth(self.coarse_smooth)
        out = ctypes.c_void_p()
        from .backend import ptr

        try:
            status = self.kernels.lib.clb_solve_loop_create(
                ctypes.byref(h.struct), ptr(self.correction), ptr(self.residual), ptr(self.direction[0]),
                ptr(self.direction[1]), ptr(self.p64[0]), ptr(self.p64[1]), ptr(self.rhs), ptr(self.fcg_state),
                ptr(self.fcg_partials), ptr(h.partials), ptr(h.norms), 0 if self.method == "fcg" else 1,
                self.pre_smooth, self.post_smooth, self.coarse_iterations, float(tol), self.max_cycles,
                ptr(self.loop_cycles), ptr(self.loop_history), int(self.loop_history.numel()), ctypes.byref(out))
        finally:
            h.struct.sweep[0] = kind0
        if status != 0:  # the host loop stays in use
            self.loop_error = (self.kernels.lib.clb_last_error() or b"").decode(errors="replace")
            return
        self._loop = out
        self._loop_key = self._key(tol)
        self.loop_launches = int(self.kernels.lib.clb_solve_loop_launches(out))

    def _run_loop(self, stats: SolveStats) -> float:
        """Runs the loop graph from the prepared state (buffer 0); returns the final relative residual."""
        k = self.kernels
        k._check(k.lib.clb_solve_loop_launch(self._loop, ptr_of(self.loop_cycles), k.stream_handle(None)),
                 "clb_solve_loop_launch")
        host = self._loop_host
        host[0:1].copy_(self.loop_cycles.to(torch.float64), non_blocking=True)
        host[1:].copy_(self.loop_history, non_blocking=True)
        torch.cuda.current_stream(k.device).synchronize()
        cycles = int(host[0])
        stats.cycles = cycles
        hist = [float(x) for x in host[2 : 2 + cycles]]  # history[1..cycles]
        stats.history.extend(hist)
        self.cur = cycles % 2
        self.graph_replays += cycles
        self.loop_refinements += cycles
        return hist[-1] if hist else stats.history[0]

    def release_loop(self) -> None:
        """Destroys the loop graph (it is rebuilt on the next solve that needs it)."""
        if self._loop is not None:
            self.kernels.lib.clb_solve_loop_destroy(self._loop)
            self._loop = None
            self._loop_key = None

    def __del__(self):
        try:
            self.release_loop()
        except Exception:
            pass
