"""FLIP timestep driver (mirrors Solver/Kernel/solver.py).

``FlipSolver`` owns one scene's device buffers and advances it with the reference's stage order
(solver.py:308-510):

 1. particle_to_grid: count, scan, stable sort, gather -> u, v, w, fluid_fraction
 2. grid_obstacle_bc (+ extrapolation) and grid_domain_bc
 3. update_velocity into the work buffers, then swap (u_work keeps the post-BC P2G field)
 4. grid_domain_bc and grid_obstacle_bc
 5. pressure solve (rhs, operator, W-cycles, Neumann ghost copy)
 6. pressure_correction, grid_domain_bc, grid_obstacle_bc
 7. grid_to_particle, previous-position copy, advection, particle domain and obstacle BCs

Steps 7's five passes run as one fused kernel; step 5 runs on the packed multigrid hierarchy.
With no collider the obstacle passes are skipped (they are exact no-ops on an empty mask).

``solver(config)`` is the reference's top-level entry (solver.py:22-531): config parsing,
voxelised static masks, host seeding, the time loop with cancellation, the particle cache and the
stats messages.
"""

from __future__ import annotations

import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import boundary_conditions, output, particles as particle_methods, source_particles, velocity_update
from . import voxelise_mesh
from .backend import Backend, default_backend
from .pressure_solve import PressureSolver, SolveStats, pressure_correction

FIELD_DTYPE = np.float32


@dataclass
class StepOptions:
    """Per-step numerical options. The defaults are the reference's semantics (pure FLIP, a fixed
    number of W-cycles); ``tol`` switches the pressure solve to mixed-precision iterative
    refinement to that relative residual."""

    flip_ratio: float = 1.0
    num_vcycles: int = 1
    tol: float | None = None
    gravity: tuple[float, float, float] = (0.0, 0.0, -9.81)
    force: tuple[float, float, float] = (0.0, 0.0, 0.0)
    rho: float = 1000.0
    nu: float = 1.0e-6
    use_graph: bool = True
    warm_start: object = None  # callable proposing an initial pressure (learned.LearnedWarmStart)
    method: str = "fcg"  # tolerance-mode iteration: "fcg" (W-cycle preconditioned CG) or "refine"
    coarse_fp16: bool = False  # tolerance mode: store the coarse levels of at most 64^3 cells in FP16
    # tolerance mode: red-black iterations of each coarsest-level solve in the W-cycle preconditioner
    # beyond its pre-smoothing (the reference's fixed-cycle W-cycle uses 64, multigrid.py defaults)
    coarse_iterations: int = 64
    # tolerance mode: red-black iterations before / after the coarse-grid correction in the W-cycle
    # preconditioner (the reference's 2 and 4)
    pre_smooth: int = 2
    post_smooth: int = 4
    # tolerance mode: the factor of every correction the W-cycle preconditioner prolongs (1: the
    # reference's piecewise-constant prolongation; about 1.7 needs far fewer cycles, see PressureSolver)
    prolong_scale: float = 1.0
    # tolerance mode: (pre, post) smoothing counts of levels >= 1 in the W-cycle preconditioner (None: the
    # pre_smooth / post_smooth above on every level, the reference)
    coarse_smooth: tuple | None = None
    revoxelise: bool = False  # voxelise the colliders again at every step (moving or deforming meshes)
    # P2G gather: "exact" (the reference's summation order, bit for bit), "tiled" (each particle visited
    # once; equal to float rounding) or "auto" (exact in the reference's fixed-cycle mode, tiled when
    # the pressure is solved to a tolerance)
    p2g: str = "auto"

    def tiled_p2g(self) -> bool:
        if self.p2g not in ("auto", "exact", "tiled"):
            raise ValueError(f"p2g must be 'auto', 'exact' or 'tiled', not {self.p2g!r}")
        return self.p2g == "tiled" or (self.p2g == "auto" and self.tol is not None)


class FlipSolver:
    """Device state and timestep of one FLIP scene on one GPU."""

    def __init__(self, kernels: Backend, grid_shape, dx: float, positions, velocities, obstacle=None,
                 dt: float = 1.0 / 240.0, options: StepOptions | None = None, particles_per_cell: int = 8,
                 min_size: int = 8, capacity: int | None = None, colliders=None, origin=(0.0, 0.0, 0.0),
                 collider_motion=None):
        self.kernels = kernels
        self.device = kernels.device
        self.grid_shape = tuple(int(s) for s in grid_shape)
        self.dx = float(dx)
        self.dt = float(dt)
        self.options = options or StepOptions()
        self.particles_per_cell = particles_per_cell
        positions = torch.as_tensor(np.ascontiguousarray(positions, dtype=np.float32)).reshape(-1, 3)
        velocities = torch.as_tensor(np.ascontiguousarray(velocities, dtype=np.float32)).reshape(-1, 3)
        self.n = int(positions.shape[0])
        cap = max(1, int(capacity or self.n))
        dev = self.device
        self.particles = torch.zeros((cap, 3), dtype=torch.float32, device=dev)
        self.particle_velocity = torch.zeros((cap, 3), dtype=torch.float32, device=dev)
        self.particles[: self.n].copy_(positions)
        self.particle_velocity[: self.n].copy_(velocities)
        (self.particle_work, self.particle_velocity_work, self.bin_counts, self.scan_outputs,
         self.scan_sums) = particle_methods.create_particle_sort_buffers(kernels, self.grid_shape, cap)
        grid = lambda: torch.zeros(self.grid_shape, dtype=torch.float32, device=dev)  # noqa: E731
        self.u, self.v, self.w = grid(), grid(), grid()
        self.u_work, self.v_work, self.w_work = grid(), grid(), grid()
        self.fluid_fraction = grid()
        self.pressure = grid()
        self.obstacle = None
        if obstacle is not None:
            ob = torch.as_tensor(np.ascontiguousarray(obstacle, dtype=np.uint8)) if isinstance(obstacle, np.ndarray) \
                else obstacle
            if bool(ob.any()):
                self.obstacle = ob.to(dev).contiguous()
        # collider meshes (world-space float32 triangles) for per-step voxelisation
        self.colliders = [torch.as_tensor(np.ascontiguousarray(t, dtype=np.float32)).to(dev) for t in (colliders or [])]
        self.origin = tuple(float(o) for o in origin)
        # a rigid motion of the colliders (colliders.RigidMotion; no counterpart in the reference): every
        # step voxelises them at their pose and uses the solid's velocity in the obstacle conditions
        self.collider_motion = collider_motion
        self._collider_rest = [np.ascontiguousarray(t, dtype=np.float32) for t in (colliders or [])]
        self._motion = None  # this step's motion parameters (grid-local), set by pre_solve
        if collider_motion is not None and not self.colliders:
            raise ValueError("collider_motion needs the collider meshes (colliders=...)")
        if self.colliders and self.obstacle is None:
            self.obstacle = torch.zeros(self.grid_shape, dtype=torch.uint8, device=dev)
        self.pressure_solver = PressureSolver(kernels, self.grid_shape, self.dx, min_size=min_size,
                                              method=self.options.method, coarse_fp16=self.options.coarse_fp16,
                                              coarse_iterations=self.options.coarse_iterations,
                                              pre_smooth=self.options.pre_smooth,
                                              post_smooth=self.options.post_smooth,
                                              prolong_scale=self.options.prolong_scale,
                                              coarse_smooth=self.options.coarse_smooth)
        self.last_solve: SolveStats | None = None
        self.steps_done = 0

    # -- the step --------------------------------------------------------------------------------
    def ensure_capacity(self, count: int) -> None:
        """Grow the particle buffers to hold ``count`` particles (by 1.5x at least, as
        solver.py:290-303 grows its buffers), keeping the current particles."""
        cap = self.particles.shape[0]
        if count <= cap:
            return
        new_cap = max(int(count), (cap * 3) // 2)
        for name in ("particles", "particle_velocity"):
            old = getattr(self, name)
            fresh = torch.zeros((new_cap, 3), dtype=torch.float32, device=self.device)
            fresh[: self.n].copy_(old[: self.n])
            setattr(self, name, fresh)
        (self.particle_work, self.particle_velocity_work, self.bin_counts, self.scan_outputs,
         self.scan_sums) = particle_methods.create_particle_sort_buffers(self.kernels, self.grid_shape, new_cap)

    def voxelise_colliders(self, queue=None) -> None:
        """Rebuild the obstacle mask from the collider meshes (voxelise_mesh.py:111-135 per mesh)."""
        self.obstacle.zero_()
        for tris in self.colliders:
            voxelise_mesh.voxelise_triangles(self.kernels, queue, tris, self.obstacle, self.grid_shape, self.dx,
                                             self.origin)

    def pre_solve(self, queue=None) -> None:
        """Stages 1-4: P2G, grid BCs, forces, BCs (everything before the pressure solve)."""
        k, o, gs = self.kernels, self.options, self.grid_shape
        self._motion = None
        if self.collider_motion is not None:
            # the pose at the step's start time; the rest triangles moved on the host (float64, rounded
            # once), voxelised on the device
            t = self.steps_done * self.dt
            for dev_tris, rest in zip(self.colliders, self._collider_rest):
                dev_tris.copy_(torch.from_numpy(self.collider_motion.transform(rest, t)))
            self.voxelise_colliders(queue)
            self._motion = self.collider_motion.parameters(t, self.origin)
        elif o.revoxelise and self.colliders:
            self.voxelise_colliders(queue)
        (self.particles, self.particle_velocity, self.particle_work, self.particle_velocity_work,
         _, self.fluid_fraction) = particle_methods.particle_to_grid(
            k, queue, self.particles, self.particle_velocity, self.particle_work, self.particle_velocity_work,
            (self.u, self.v, self.w), self.bin_counts, self.scan_outputs, self.scan_sums, self.fluid_fraction, self.n,
            gs, self.dx, self.particles_per_cell, tiled=o.tiled_p2g())
        vel = (self.u, self.v, self.w)
        if self.obstacle is not None:
            boundary_conditions.grid_obstacle_bc(k, queue, vel, self.fluid_fraction, self.obstacle, gs,
                                                 self._motion, self.dx)
        boundary_conditions.grid_domain_bc(k, queue, vel, gs)
        velocity_update.update_velocity(k, queue, vel, (self.u_work, self.v_work, self.w_work), self.fluid_fraction,
                                        o.gravity, *o.force, o.rho, o.nu, self.dx, self.dt, gs)
        self.u, self.u_work = self.u_work, self.u
        self.v, self.v_work = self.v_work, self.v
        self.w, self.w_work = self.w_work, self.w
        vel = (self.u, self.v, self.w)
        boundary_conditions.grid_domain_bc(k, queue, vel, gs)
        if self.obstacle is not None:
            boundary_conditions.grid_obstacle_bc(k, queue, vel, self.fluid_fraction, self.obstacle, gs,
                                                 self._motion, self.dx)

    def solve(self, tol: float | None = None, num_vcycles: int | None = None) -> SolveStats:
        """Stage 5: the pressure solve, warm-started from the previous step's pressure."""
        o = self.options
        stats = self.pressure_solver.solve((self.u, self.v, self.w), self.fluid_fraction, self.pressure, self.dt,
                                           o.rho, num_vcycles=o.num_vcycles if num_vcycles is None else num_vcycles,
                                           tol=o.tol if tol is None else tol, use_graph=o.use_graph,
                                           warm_start=o.warm_start, solid=self.obstacle)
        self.last_solve = stats
        return stats

    def post_solve(self, queue=None, piece_bounds=None, piece_done=None) -> None:
        """Stages 6-7: projection, BCs and the fused particle update. ``piece_bounds`` (ascending
        particle indices from 0 to n) splits the particle update into one launch per piece, each
        followed by ``piece_done(piece)`` (the update of one particle does not depend on another's)."""
        k, o, gs = self.kernels, self.options, self.grid_shape
        vel = (self.u, self.v, self.w)
        ps = self.pressure_solver
        if ps.solved64:
            # a tolerance-mode solve: project with the FP64 pressure that meets the tolerance
            k.call("clb_pressure_correction_f64", *vel, ps.pressure64, float(np.float32(self.dt / o.rho)),
                   float(np.float32(1.0 / self.dx)), *gs, stream=queue)
        else:
            pressure_correction(k, queue, vel, self.pressure, self.dx, self.dt, o.rho, gs)
        boundary_conditions.grid_domain_bc(k, queue, vel, gs)
        if self.obstacle is not None:
            boundary_conditions.grid_obstacle_bc(k, queue, vel, self.fluid_fraction, self.obstacle, gs,
                                                 self._motion, self.dx)
        if piece_bounds is None:
            # the particles are still sorted by bin from this step's P2G: the tiled update (same values)
            particle_methods.particle_update(k, queue, self.particles, self.particle_velocity, vel,
                                             (self.u_work, self.v_work, self.w_work), self.obstacle, self.n, gs,
                                             self.dx, self.dt, o.flip_ratio, motion=self._motion,
                                             bins=(self.scan_outputs[0], self.bin_counts))
            return
        for c in range(len(piece_bounds) - 1):
            a, b = piece_bounds[c], piece_bounds[c + 1]
            if b > a:
                particle_methods.particle_update(k, queue, self.particles[a:b], self.particle_velocity[a:b], vel,
                                                 (self.u_work, self.v_work, self.w_work), self.obstacle, b - a, gs,
                                                 self.dx, self.dt, o.flip_ratio, motion=self._motion)
            piece_done(c)

    def step(self) -> SolveStats:
        if self.n == 0:
            self.steps_done += 1
            return SolveStats()
        self.pre_solve()
        stats = self.solve()
        self.post_solve()
        self.steps_done += 1
        return stats

    def step_host(self, positions: torch.Tensor, velocities: torch.Tensor, chunks: int = 8) -> SolveStats:
        """One step with the particle state making the host round trip that solver.py:252-306 makes
        every step: ``positions`` and ``velocities`` (pinned float32 host tensors of shape (n, 3)) are
        uploaded, the step runs, and the new state is downloaded into the same tensors.

        The copies run in ``chunks`` pieces on two copy streams. The step's last stage, the particle
        update, runs one launch per piece, and a piece's download starts once its update is done. In
        back-to-back calls a piece's upload waits only for the previous call's download of that piece,
        so the download of one call and the upload of the next overlap piece by piece: the link carries
        both directions at once. The call returns once the work is enqueued: the host tensors hold the
        new state after ``torch.cuda.synchronize()``. Work on the current stream after the call waits
        for the download; between calls, the caller synchronises before it reads or changes the host
        tensors or the particle state by other means."""
        n = self.n
        for name, t in (("positions", positions), ("velocities", velocities)):
            if t.device.type != "cpu" or not t.is_pinned() or t.dtype != torch.float32 or tuple(t.shape) != (n, 3) \
                    or not t.is_contiguous():
                raise ValueError(f"step_host: {name} must be a contiguous pinned float32 host tensor of shape ({n}, 3)")
        chunks = max(1, min(int(chunks), max(n, 1)))
        if getattr(self, "_host_streams", None) is None:
            self._host_streams = (torch.cuda.Stream(self.device), torch.cuda.Stream(self.device))
            self._host_events: list = []
        up, down = self._host_streams
        compute = torch.cuda.current_stream(self.device)
        bounds = [(n * c) // chunks for c in range(chunks + 1)]
        previous = self._host_events if len(self._host_events) == chunks else None
        if previous is None:
            # the first call (or another piece count): the upload waits for all work so far
            up.wait_stream(compute)
            up.wait_stream(down)
        with torch.cuda.stream(up):
            for c in range(chunks):
                a, b = bounds[c], bounds[c + 1]
                if previous is not None:
                    up.wait_event(previous[c])
                self.particles[a:b].copy_(positions[a:b], non_blocking=True)
                self.particle_velocity[a:b].copy_(velocities[a:b], non_blocking=True)
        compute.wait_stream(up)
        updated = []

        def piece_done(c: int) -> None:
            ev = torch.cuda.Event()
            ev.record(compute)
            updated.append(ev)

        if n == 0:
            stats = self.step()
        else:
            self.pre_solve()
            stats = self.solve()
            self.post_solve(piece_bounds=bounds, piece_done=piece_done)
            self.steps_done += 1
        if self.n != n:
            raise RuntimeError("step_host: the step changed the particle count; use step() with sources")
        if len(updated) != chunks:
            down.wait_stream(compute)
        events = []
        with torch.cuda.stream(down):
            for c in range(chunks):
                a, b = bounds[c], bounds[c + 1]
                if len(updated) == chunks:
                    down.wait_event(updated[c])
                positions[a:b].copy_(self.particles[a:b], non_blocking=True)
                velocities[a:b].copy_(self.particle_velocity[a:b], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(down)
                events.append(ev)
        self._host_events = events
        compute.wait_stream(down)
        return stats

    # -- host views -------------------------------------------------------------------------------
    def positions(self) -> np.ndarray:
        return self.particles[: self.n].cpu().numpy()

    def velocities(self) -> np.ndarray:
        return self.particle_velocity[: self.n].cpu().numpy()


def scene_solver(kernels: Backend, scene, options: StepOptions | None = None) -> FlipSolver:
    """Build a FlipSolver for a ``scenes.Scene``: voxelise its colliders on the device, seed its
    particles on the host around the solid cells, upload."""
    obstacle = torch.zeros(scene.grid_shape, dtype=torch.uint8, device=kernels.device)
    for tris in scene.obstacles:
        voxelise_mesh.voxelise_triangles(kernels, None, tris, obstacle, scene.grid_shape, scene.dx, scene.origin)
    from .scenes import seed_particles

    positions, velocities = seed_particles(scene, obstacle.cpu().numpy())
    opts = options or StepOptions(flip_ratio=scene.flip_ratio, gravity=scene.gravity, rho=scene.rho, nu=scene.nu)
    return FlipSolver(kernels, scene.grid_shape, scene.dx, positions, velocities, obstacle=obstacle, dt=scene.dt,
                      options=opts, particles_per_cell=scene.particles_per_cell, min_size=scene.min_size,
                      colliders=scene.obstacles, origin=scene.origin)


def moving_colliders(simulation: dict):
    """The obstacles' world triangles and their rigid motion when the config gives one (an obstacle's
    "motion": {"velocity", "angular_velocity", "pivot"}; no counterpart in the reference). All
    obstacles of a scene then move together: one motion, given on every obstacle."""
    from .colliders import RigidMotion

    obstacles = simulation.get("obstacles") or ()
    motions = [RigidMotion.from_config(o.get("motion")) for o in obstacles]
    if all(m is None for m in motions):
        return [], None
    if any(m != motions[0] for m in motions):
        raise ValueError("moving obstacles: every obstacle of a scene must give the same motion (one rigid body)")
    bake_path = simulation.get("output_path", ".")
    tris = [voxelise_mesh._entry_triangles(entry, bake_path) for o in obstacles for entry in o.get("geometry_inputs") or ()]
    return [t for t in tris if t.size], motions[0]


# ------------------------------------------------------------------------------------------------
# solver(config): the reference's entry point (solver.py:22-531)
# ------------------------------------------------------------------------------------------------
def solver(config: dict, timings=None) -> None:
    from .general.main import emit_message

    simulation = config.get("simulation") or {}
    settings = simulation.get("settings") or {}
    kernels = default_backend()
    domain = simulation.get("domain") or {}
    domain_size = domain.get("size") or {}
    physics = simulation.get("physics") or {}
    water = physics.get("water") or {}
    output_dir = Path(simulation["output_path"]).expanduser().resolve()
    cancel_event = (config.get("meta") or {}).get("cancel_event")

    start_frame = int(settings.get("start_frame", 1))
    end_frame = int(settings.get("end_frame", 250))
    fps = int(settings.get("fps", 24))
    substeps = max(0, int(settings.get("substeps", 1)))
    steps_per_frame = substeps + 1
    total_frames = max(0, end_frame - start_frame)
    total_solver_steps = total_frames * steps_per_frame
    dt = 1.0 / (fps * steps_per_frame)

    delta = float(domain["resolution"])
    grid_shape = (int(float(domain_size["x"]) / delta), int(float(domain_size["y"]) / delta),
                  int(float(domain_size["z"]) / delta))
    rho_water = float(water["density"])
    nu_water = float(water["viscosity"])
    options = StepOptions(
        flip_ratio=float(settings.get("flip_ratio", 1.0)),
        num_vcycles=max(1, int(settings.get("iterations", 1))),
        tol=settings.get("tolerance"),
        gravity=tuple(settings.get("gravity", (0.0, 0.0, -9.81))),
        rho=rho_water,
        nu=nu_water,
    )

    sources_dev, obstacle_mask = voxelise_mesh.build_static_masks(kernels, None, kernels, simulation, grid_shape,
                                                                  delta)
    # the reference seeds on the host from default_rng(0) (solver.py:146-158); the device sources
    # draw the same stream, so the particles equal the reference's without leaving the GPU
    rng = np.random.default_rng(0)
    empty = np.empty((0, 3), dtype=FIELD_DTYPE)
    colliders, motion = moving_colliders(simulation)
    size = domain_size
    origin = (-0.5 * float(size["x"]), -0.5 * float(size["y"]), 0.0)
    sim = FlipSolver(kernels, grid_shape, delta, empty, empty, obstacle=obstacle_mask, dt=dt, options=options,
                     particles_per_cell=8, colliders=colliders if motion is not None else None, origin=origin,
                     collider_motion=motion)
    source_particles.DeviceSources(kernels, sources_dev, obstacle_mask, grid_shape, delta, rng,
                                   initial=True).apply(sim)
    device_sources = source_particles.DeviceSources(kernels, sources_dev, obstacle_mask, grid_shape, delta, rng)

    output_dir.mkdir(parents=True, exist_ok=True)
    cache = output.create_cache(output_dir, fps=fps, start_frame=start_frame, end_frame=end_frame)
    writer = output.create_output(cache)
    try:
        output.submit_output(writer, particles=sim.particles, particle_count=sim.n, frame=start_frame)
        emit_message({"type": "stats", "frame": 0, "total_frames": total_frames, "particle_count": sim.n})
        dynamic = any(source.get("type") in {"INFLOW", "OUTFLOW"} for source in sources_dev)
        for solver_step in range(total_solver_steps):
            if cancel_event is not None and cancel_event.is_set():
                print("Bake cancellation requested. Stopping the simulation cleanly...")
                break
            output_frame = (solver_step + 1) // steps_per_frame
            substep_index = solver_step % steps_per_frame
            if dynamic:
                # the reference's per-step host round trip (solver.py:252-306), on the device
                device_sources.apply(sim)
            t0 = time.perf_counter()
            stats = sim.step()
            if substep_index == steps_per_frame - 1:
                output.submit_output(writer, particles=sim.particles, particle_count=sim.n,
                                     frame=start_frame + output_frame)
                emit_message({"type": "stats", "frame": output_frame, "total_frames": total_frames,
                              "particle_count": sim.n, "solve": {"cycles": stats.cycles,
                                                                 "rel_residual": stats.rel_residual,
                                                                 "ms": (time.perf_counter() - t0) * 1e3}})
    finally:
        output.close_output(writer)
