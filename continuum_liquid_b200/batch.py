"""Batched scenes: many independent FLIP scenes of different grid sizes advancing together, one launch
per stage (no counterpart in the reference, which bakes one scene at a time).

Every grid field of the batch holds the scenes' grids back to back (level 0 for the simulation
fields, one array per multigrid level), all particles are one array, and each stage is one
``clb_batch_*`` launch whose threads find their scene from a prefix table (csrc/batch.cuh). In
reference mode (``tol=None``) each scene's values equal a single-scene ``FlipSolver`` run bit for
bit; in tolerance mode every scene is solved by the flexible CG with FP64 accumulation until every
scene's relative residual is at most ``tol``.

The step is captured in CUDA graphs: everything up to the initial residual (one graph), one
flexible-CG iteration per ping-pong direction (two graphs, replayed between host checks of the
per-scene residuals) and the projection and particle update (one graph).
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import voxelise_mesh
from .backend import BATCH_MAX_SCENES, MG_MAX_LEVELS, Backend, Batch, BatchList, BatchScene
from .multigrid import COARSE_SMOOTH_ITERATIONS, POST_SMOOTH, PRE_SMOOTH, level_shapes_for
from .pressure_solve import FIELD_DTYPE, SolveStats
from .scenes import Scene, seed_particles

F32 = np.float32
BOTTOM_SMEM_LIMIT = 220 * 1024  # csrc/clb200.cu kBottomSmemLimit
BOTTOM_THREADS, BOTTOM_BTHREADS, BOTTOM_MAX_A, BOTTOM_MAX_B = 512, 256, 8, 4  # csrc/mg_bottom.cuh


def _pad16(x: int) -> int:
    return (x + 15) & ~15


def bottom_plan(shapes) -> tuple[int, int, int, int]:
    """(bottom level, register tiles ka, kb, shared-memory bytes) of the single-block bottom visit for a
    level pyramid, with the rule of csrc/clb200.cu bottom_visit; level -1 when it does not apply."""
    levels = len(shapes)
    level = levels - 2
    if level < 1:
        return -1, 0, 0, 0
    a, b = shapes[level], shapes[level + 1]
    ca, cb = int(np.prod(a)), int(np.prod(b))
    sa, sb = colour_slots(a), colour_slots(b)
    smem = _pad16(ca * 4) * 2 + ca * 16 + _pad16(cb * 4) + cb * 16 + _pad16((ca + cb + 8) * 4)
    if smem > BOTTOM_SMEM_LIMIT or sb > BOTTOM_MAX_B * BOTTOM_BTHREADS or sa > BOTTOM_MAX_A * BOTTOM_THREADS:
        return -1, 0, 0, 0
    return level, -(-sa // BOTTOM_THREADS), -(-sb // BOTTOM_BTHREADS), smem


def colour_slots(shape) -> int:
    """Cells of one colour a thread set must cover on a level (csrc/mg_bottom.cuh colour_slots)."""
    return (shape[0] - 2) * (shape[1] - 2) * ((shape[2] - 1) // 2)


@dataclass
class BatchStats:
    cycles: int
    rel_residual: list  # per scene (tolerance mode)
    history: list


class BatchedFlip:
    """Device state and timestep of a batch of scenes (all with the same dt, rho, nu, gravity)."""

    def __init__(self, kernels: Backend, scenes: list[Scene], flip_ratio: float | None = None, tol: float | None = 1e-6,
                 num_vcycles: int = 1, reduce_blocks: int = 32, sweep0: int = 1, use_graph: bool = True,
                 max_cycles: int = 100, coarse_iterations: int = COARSE_SMOOTH_ITERATIONS,
                 pre_smooth: int = PRE_SMOOTH, post_smooth: int = POST_SMOOTH, tiled_p2g: bool | None = None,
                 prolong_scale: float = 1.0, coarse_smooth=None):
        if not 1 <= len(scenes) <= BATCH_MAX_SCENES:
            raise ValueError(f"a batch holds 1..{BATCH_MAX_SCENES} scenes, got {len(scenes)}")
        first = scenes[0]
        for s in scenes:
            if (s.dt, s.rho, s.nu, tuple(s.gravity)) != (first.dt, first.rho, first.nu, tuple(first.gravity)):
                raise ValueError("the scenes of a batch share dt, rho, nu and gravity")
        self.k = kernels
        self.scenes = scenes
        self.S = len(scenes)
        self.dt, self.rho, self.nu, self.gravity = first.dt, first.rho, first.nu, tuple(first.gravity)
        self.flip_ratio = first.flip_ratio if flip_ratio is None else float(flip_ratio)
        self.tol, self.num_vcycles, self.max_cycles = tol, int(num_vcycles), int(max_cycles)
        # coarsest-level iterations of the tolerance mode's W-cycle preconditioner (fixed-cycle mode: 64)
        self.coarse_iterations = int(coarse_iterations)
        # smoothing sweeps per level of the tolerance mode's W-cycle preconditioner (fixed-cycle mode:
        # the reference's 2 and 4)
        self.pre_smooth, self.post_smooth = int(pre_smooth), int(post_smooth)
        if self.pre_smooth < 0 or self.post_smooth < 0 or self.pre_smooth + self.post_smooth == 0:
            raise ValueError("pre_smooth and post_smooth must be >= 0 and not both 0")
        # factor of every correction the tolerance mode's W-cycle prolongs (PressureSolver.prolong_scale;
        # fixed-cycle mode: 1, the reference's prolongation)
        self.prolong_scale = float(prolong_scale)
        if not self.prolong_scale > 0.0:
            raise ValueError("prolong_scale must be > 0")
        # smoothing counts (pre, post) of levels >= 1 (PressureSolver.coarse_smooth; None: every level as 0)
        self.coarse_smooth = None if coarse_smooth is None else tuple(int(x) for x in coarse_smooth)
        self.ppc = first.particles_per_cell
        self.use_graph = use_graph
        dev = kernels.device
        self.shapes = [[tuple(s.grid_shape), *level_shapes_for(s.grid_shape, s.min_size)] for s in scenes]
        self.levels = max(len(sh) for sh in self.shapes)
        if self.levels > MG_MAX_LEVELS:
            raise ValueError("too many multigrid levels")
        self.cells = [[int(np.prod(sh[l])) if l < len(sh) else 0 for l in range(self.levels)] for sh in self.shapes]
        self.level_total = [sum(c[l] for c in self.cells) for l in range(self.levels)]
        self.base = [[0] * self.levels for _ in scenes]
        for l in range(self.levels):
            acc = 0
            for s in range(self.S):
                self.base[s][l] = acc
                acc += self.cells[s][l]
        self.plans = [bottom_plan(sh) for sh in self.shapes]
        C0 = self.level_total[0]
        self.C0 = C0

        # ---- colliders and particles ----------------------------------------------------------------
        grid = lambda dtype=torch.float32: torch.zeros(C0, dtype=dtype, device=dev)  # noqa: E731
        self.obstacle = grid(torch.uint8)
        positions, velocities = [], []
        for s, sc in enumerate(scenes):
            view = self.scene_view(self.obstacle, s)
            for tris in sc.obstacles:
                voxelise_mesh.voxelise_triangles(kernels, None, tris, view, sc.grid_shape, sc.dx, sc.origin)
            pos, vel = seed_particles(sc, view.cpu().numpy())
            positions.append(pos)
            velocities.append(vel)
        self.counts = [len(p) for p in positions]
        self.particle_base = np.concatenate([[0], np.cumsum(self.counts)[:-1]]).astype(np.int64)
        self.n = int(sum(self.counts))
        pos = torch.from_numpy(np.concatenate(positions).reshape(-1, 3)).to(dev)
        vel = torch.from_numpy(np.concatenate(velocities).reshape(-1, 3)).to(dev)
        self.particles, self.particle_velocity = pos.contiguous(), vel.contiguous()
        self.particle_work = torch.empty_like(self.particles)
        self.particle_velocity_work = torch.empty_like(self.particle_velocity)
        ni = max(1, self.n)
        self.keys, self.ranks, self.perm, self.slot_keys = (torch.empty(ni, dtype=torch.int32, device=dev)
                                                            for _ in range(4))
        self.scan = torch.empty(kernels.scan_scratch_bytes(C0), dtype=torch.uint8, device=dev)

        # ---- fields -----------------------------------------------------------------------------------
        self.u, self.v, self.w = grid(), grid(), grid()
        self.u_work, self.v_work, self.w_work = grid(), grid(), grid()
        self.fluid_fraction, self.pressure, self.rhs = grid(), grid(), grid()
        self.residual, self.correction = grid(), grid()
        self.bin_counts, self.bin_offsets = grid(torch.int32), grid(torch.int32)
        self.op0 = grid(torch.uint8)
        self.p64 = [grid(torch.float64) for _ in range(2)]
        self.direction = [grid() for _ in range(2)]
        self.fcg_state = torch.zeros(4 * self.S, dtype=torch.float64, device=dev)
        self.partials = torch.zeros(2 * self.S * reduce_blocks, dtype=torch.float64, device=dev)
        self.partials4 = torch.zeros(4 * self.S * reduce_blocks, dtype=torch.float64, device=dev)
        self.norms = torch.zeros(2 * self.S, dtype=torch.float64, device=dev)
        self.norms_host = torch.zeros(2 * self.S, dtype=torch.float64, pin_memory=True)
        self.lp, self.lb, self.lmask, self.lop = [None], [None], [None], [None]
        for l in range(1, self.levels):
            t = self.level_total[l]
            self.lp.append(torch.zeros(max(t, 1), dtype=torch.float32, device=dev))
            self.lb.append(torch.zeros(max(t, 1), dtype=torch.float32, device=dev))
            self.lmask.append(torch.zeros(max(t, 1), dtype=torch.uint8, device=dev))
            self.lop.append(torch.zeros((max(t, 1), 4), dtype=torch.float32, device=dev))

        # ---- geometry table and launch lists --------------------------------------------------------------
        self._keep: list = []
        geom = (BatchScene * self.S)()
        for s, sc in enumerate(scenes):
            g = geom[s]
            g.levels = len(self.shapes[s])
            g.bottom = self.plans[s][0]
            for l, sh in enumerate(self.shapes[s]):
                for a in range(3):
                    g.shape[l][a] = sh[a]
                g.base[l] = self.base[s][l]
            g.particle_base = int(self.particle_base[s])
            g.particles = self.counts[s]
            dx = float(sc.dx)
            g.delta = float(FIELD_DTYPE(dx))
            g.inv_dx = float(FIELD_DTYPE(1.0 / dx))
            g.inv_dx2 = float(FIELD_DTYPE(1.0 / (dx * dx)))
            g.rho_over_dt = float(FIELD_DTYPE(float(sc.rho) / float(sc.dt)))
            g.dt_over_rho = float(FIELD_DTYPE(float(sc.dt) / float(sc.rho)))
            g.lower = float(FIELD_DTYPE(1.001 * dx))
            for a in range(3):
                g.upper[a] = float(FIELD_DTYPE((sc.grid_shape[a] - 1.001) * dx))
        self.geom_host = geom
        self.geom_dev = torch.frombuffer(bytearray(bytes(geom)), dtype=torch.uint8).to(dev)
        b = Batch()
        b.scenes = self.S
        b.levels = self.levels
        b.geom = self.geom_dev.data_ptr()
        b.geom_host = ctypes.addressof(geom)
        b.particles = self._list(range(self.S), self.counts)
        L = [len(sh) for sh in self.shapes]
        bottom = [p[0] for p in self.plans]
        for l in range(self.levels):
            having = [s for s in range(self.S) if l < L[s]]
            b.cells[l] = self._list(having, [self.cells[s][l] for s in having])
            rec = [s for s in range(self.S) if l < L[s] - 1 and (bottom[s] < 0 or l < bottom[s])]
            b.recurse[l] = self._list(rec, [self.cells[s][l] for s in rec])
            b.recurse_coarse[l] = self._list(rec, [self.cells[s][l + 1] for s in rec] if l + 1 < self.levels else [])
            bot = [s for s in range(self.S) if bottom[s] == l]
            b.bottom[l] = self._list(bot, [1] * len(bot))
            co = [s for s in range(self.S) if bottom[s] < 0 and l == L[s] - 1]
            b.coarse[l] = self._list(co, [1] * len(co))
        rec0 = [s for s in range(self.S) if 0 < L[s] - 1 and (bottom[s] < 0 or 0 < bottom[s])]
        vec = 4 if all(self.shapes[s][0][2] % 4 == 0 and self.base[s][0] % 4 == 0 for s in rec0) else 1
        blocks = [-(-self.shapes[s][0][2] // (32 * vec)) * -(-self.shapes[s][0][1] // 4) * self.shapes[s][0][0]
                  for s in rec0]
        b.colour0 = self._list(rec0, blocks)
        b.sweep0 = int(sweep0)
        b.vec0 = vec
        # P2G: the tiled scatter in tolerance mode (each particle visited once; the same values as the
        # single-scene tiled P2G), the reference-order gather in the fixed-cycle mode (None: by mode)
        b.p2g_tiled = int(tol is not None if tiled_p2g is None else bool(tiled_p2g))
        b.reduce_blocks = int(reduce_blocks)
        used = [p for p in self.plans if p[0] >= 0]
        b.bottom_ka = max((p[1] for p in used), default=0)
        b.bottom_kb = max((p[2] for p in used), default=0)
        b.bottom_smem = max((p[3] for p in used), default=0)
        b.op0 = self.op0.data_ptr()
        for l in range(1, self.levels):
            b.p[l] = self.lp[l].data_ptr()
            b.b[l] = self.lb[l].data_ptr()
            b.mask[l] = self.lmask[l].data_ptr()
            b.op[l] = self.lop[l].data_ptr()
        self.batch = b
        self.steps_done = 0
        self._graphs: dict = {}
        self.graph_replays = 0

    # -- helpers ----------------------------------------------------------------------------------------
    def _list(self, scenes, items) -> BatchList:
        lst = BatchList()
        scenes = list(scenes)
        lst.count = len(scenes)
        if not scenes:
            return lst
        start = np.concatenate([[0], np.cumsum(np.asarray(items, dtype=np.int64))]).astype(np.int64)
        sc = torch.tensor(scenes, dtype=torch.int32, device=self.k.device)
        st = torch.from_numpy(start).to(self.k.device)
        self._keep += [sc, st]
        lst.scene = sc.data_ptr()
        lst.start = st.data_ptr()
        lst.total = int(start[-1])
        return lst

    def scene_view(self, field: torch.Tensor, s: int, level: int = 0) -> torch.Tensor:
        """Scene s's part of a batch-wide level-0 field, shaped as its grid."""
        b, c = self.base[s][level], self.cells[s][level]
        return field[b: b + c].view(self.shapes[s][level])

    def positions(self, s: int) -> np.ndarray:
        b = int(self.particle_base[s])
        return self.particles[b: b + self.counts[s]].cpu().numpy()

    def velocities(self, s: int) -> np.ndarray:
        b = int(self.particle_base[s])
        return self.particle_velocity[b: b + self.counts[s]].cpu().numpy()

    def _call(self, name, *args):
        self.k.call_batch(name, self.batch, *args)

    # -- the step -----------------------------------------------------------------------------------------
    def _pre_work(self) -> None:
        """Stages 1-4 of every scene (solver.py:335-420): P2G, grid BCs, forces, BCs, then the pressure
        right-hand side and operators. Writes the sorted particles to the work buffers and the forced
        velocity to the velocity work buffers; ``_swap`` then exchanges the roles (no swap happens
        here, so the work can be captured in a graph and replayed)."""
        self._call("clb_batch_particle_to_grid", self.particles, self.particle_velocity, self.particle_work,
                   self.particle_velocity_work, self.u, self.v, self.w, self.fluid_fraction, self.bin_counts,
                   self.bin_offsets, self.keys, self.ranks, self.perm, self.slot_keys, self.scan,
                   int(self.scan.numel()), float(FIELD_DTYPE(1.0 / self.ppc)))
        vel = (self.u, self.v, self.w)
        self._call("clb_batch_grid_obstacle_bc", *vel, self.fluid_fraction, self.obstacle)
        self._call("clb_batch_grid_domain_bc", *vel)
        g = self.gravity
        forced = (self.u_work, self.v_work, self.w_work)
        self._call("clb_batch_update_velocity", *vel, *forced, self.fluid_fraction, float(FIELD_DTYPE(g[0])),
                   float(FIELD_DTYPE(g[1])), float(FIELD_DTYPE(g[2])), 0.0, 0.0, 0.0, float(FIELD_DTYPE(self.rho)),
                   float(FIELD_DTYPE(self.nu)), float(FIELD_DTYPE(self.dt)))
        self._call("clb_batch_grid_domain_bc", *forced)
        self._call("clb_batch_grid_obstacle_bc", *forced, self.fluid_fraction, self.obstacle)
        self._call("clb_batch_rhs_operator", *forced, self.fluid_fraction, self.rhs)

    def _swap(self) -> None:
        self.particles, self.particle_work = self.particle_work, self.particles
        self.particle_velocity, self.particle_velocity_work = self.particle_velocity_work, self.particle_velocity
        self.u, self.u_work = self.u_work, self.u
        self.v, self.v_work = self.v_work, self.v
        self.w, self.w_work = self.w_work, self.w

    def pre_solve(self) -> None:
        self._pre_work()
        self._swap()

    def _w_cycle(self, x, rhs, coarse_iterations: int = COARSE_SMOOTH_ITERATIONS, pre: int = PRE_SMOOTH,
                 post: int = POST_SMOOTH, prolong_scale: float = 1.0, coarse_smooth=None) -> None:
        # read when the W-cycle is launched or captured
        self.batch.prolong_scale = float(prolong_scale)
        self.batch.coarse_smoothing = 0 if coarse_smooth is None else 1
        if coarse_smooth is not None:
            self.batch.coarse_pre_smooth, self.batch.coarse_post_smooth = (int(x) for x in coarse_smooth)
        self._call("clb_batch_w_cycle", x, rhs, int(pre), int(post), int(coarse_iterations))

    def _init_solve(self) -> None:
        self.cur = 0
        self.direction[0].zero_()
        self.fcg_state.zero_()
        self._call("clb_batch_ir_init", self.pressure, self.p64[0])
        self._call("clb_batch_residual_norms", self.p64[0], 1, self.rhs, self.residual, self.partials, self.norms)

    def _iteration(self, src: int) -> None:
        self.correction.zero_()
        self._w_cycle(self.correction, self.residual, self.coarse_iterations, self.pre_smooth, self.post_smooth,
                      self.prolong_scale, self.coarse_smooth)
        self._call("clb_batch_fcg_dots", self.correction, self.direction[src], self.residual, self.partials4,
                   self.fcg_state)
        self._call("clb_batch_fcg_step", self.p64[src], self.correction, self.direction[src], self.p64[1 - src],
                   self.direction[1 - src], self.fcg_state, self.rhs, self.residual, self.partials, self.norms)

    def _post(self, tolerance: bool) -> None:
        vel = (self.u, self.v, self.w)
        if tolerance:
            self._call("clb_batch_ir_store", self.p64[self.cur], self.pressure)
            self._call("clb_batch_pressure_correction", *vel, self.p64[self.cur], 1)
        else:
            self._call("clb_batch_neumann_domain_bc", self.pressure)
            self._call("clb_batch_pressure_correction", *vel, self.pressure, 0)
        self._call("clb_batch_grid_domain_bc", *vel)
        self._call("clb_batch_grid_obstacle_bc", *vel, self.fluid_fraction, self.obstacle)
        self._call("clb_batch_particle_update", self.particles, self.particle_velocity, *vel, self.u_work,
                   self.v_work, self.w_work, self.obstacle, float(FIELD_DTYPE(self.flip_ratio)),
                   float(FIELD_DTYPE(self.dt)))

    def _run(self, key, fn) -> None:
        """Run fn, or replay its CUDA graph (captured on first use; buffer swaps happen outside)."""
        if not self.use_graph:
            fn()
            return
        graph = self._graphs.get(key)
        if graph is None:
            stream = torch.cuda.current_stream(self.k.device)
            side = torch.cuda.Stream(self.k.device)
            side.wait_stream(stream)
            with torch.cuda.stream(side):
                fn()  # the first use runs eagerly, then is captured without being replayed
            stream.wait_stream(side)
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                fn()
            self._graphs[key] = graph
        else:
            graph.replay()
            self.graph_replays += 1

    def _rel(self) -> np.ndarray:
        self.norms_host.copy_(self.norms, non_blocking=True)
        torch.cuda.current_stream(self.k.device).synchronize()
        v = self.norms_host.numpy().reshape(self.S, 2)
        return np.where(v[:, 1] > 0, np.sqrt(v[:, 0] / np.where(v[:, 1] > 0, v[:, 1], 1.0)), 0.0)

    def solve(self) -> BatchStats:
        if self.tol is None:
            for _ in range(self.num_vcycles):
                self._w_cycle(self.pressure, self.rhs)
            return BatchStats(self.num_vcycles, [], [])
        self._init_solve()
        rel = self._rel()
        hist = [float(rel.max())]
        cycles, rate = 0, None
        while rel.max() > self.tol and cycles < self.max_cycles:
            batch = 1
            if rate is not None and 0.0 < rate < 1.0:
                batch = max(1, int(math.ceil(math.log(self.tol / rel.max()) / math.log(rate))) - 1)
            batch = min(batch, self.max_cycles - cycles, 8)
            for _ in range(batch):
                src = self.cur
                # the ping-pong buffers are part of what is captured, so each direction has its own graph
                self._run(("it", src), lambda src=src: self._iteration(src))
                self.cur = 1 - src
            prev = rel.max()
            cycles += batch
            rel = self._rel()
            hist.append(float(rel.max()))
            rate = (rel.max() / prev) ** (1.0 / batch) if prev > 0 and cycles > 1 else None
        return BatchStats(cycles, [float(r) for r in rel], hist)

    def step(self) -> BatchStats:
        # graphs are keyed by the buffers they were captured with (the particle and velocity buffers
        # alternate between steps, the FP64 pressure between iterations)
        self._run(("pre", self.particles.data_ptr(), self.u.data_ptr()), self._pre_work)
        self._swap()
        stats = self.solve()
        tolerance = self.tol is not None
        cur = self.cur if tolerance else 0
        self._run(("post", tolerance, cur, self.particles.data_ptr(), self.u.data_ptr()),
                  lambda: self._post(tolerance))
        self.steps_done += 1
        return stats
