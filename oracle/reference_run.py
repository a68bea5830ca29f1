"""Runs the reference solver itself (Solver/General/main.py main(config)) on the host CPU and
records what it computes. Test infrastructure only: it needs the reference checkout, so it runs in
the container that holds it, where tests/golden/make_reference_golden.py turns its records into
committed fixtures.

The reference's Python host code runs unmodified against the pyopencl stand-in
(oracle/pyopencl_shim), which executes the reference's own OpenCL kernels compiled for the host by
oracle/ref_build.py. Two things are supplied from outside, because this machine lacks them:

* USD mesh loading (`voxelise_mesh.load_usdc_triangles`, which needs `pxr`): replaced by a lookup
  of the triangles the caller passes for each `mesh_file` name; the world transform, the
  voxelisation and everything after it are the reference's.
* observation: the stage functions the solver calls (`particles.particle_to_grid`,
  `pressure_solve.pressure_solve`, `particles.grid_to_particle`, `voxelise_mesh.build_static_masks`)
  are wrapped so that their inputs and results are copied out for the first `capture_steps` steps;
  the wrappers call the originals with the same arguments and return their results unchanged.
"""

from __future__ import annotations

import os
import sys
import tempfile
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
SHIM_DIR = ORACLE_DIR / "pyopencl_shim"
DEFAULT_REFERENCE = Path(os.environ.get("CLB_REFERENCE_ROOT", "/root/reference"))


def available(reference_root: Path = DEFAULT_REFERENCE) -> bool:
    return (reference_root / "Solver" / "General" / "main.py").exists()


def _import_reference(reference_root: Path):
    for path in (str(reference_root), str(SHIM_DIR)):
        if path not in sys.path:
            sys.path.insert(0, path)
    import pyopencl  # noqa: F401

    if not getattr(pyopencl, "VERSION_TEXT", "") == "host shim":
        raise RuntimeError("a real pyopencl shadows the host shim")
    from Solver.General import main as ref_main  # type: ignore
    from Solver.Kernel import particles, pressure_solve, voxelise_mesh  # type: ignore

    return ref_main, particles, pressure_solve, voxelise_mesh


def _array(buffer, dtype, count=None):
    data = buffer.bytes.view(dtype)
    return (data if count is None else data[:count]).copy()


def run(config: dict, meshes: dict[str, np.ndarray], capture_steps: int = 1,
        reference_root: Path = DEFAULT_REFERENCE) -> dict:
    """Runs main(config) of the reference. `meshes` maps each geometry entry's `mesh_file` to its
    (T, 3, 3) float32 triangles in object space. Returns {"frames": [(N, 3) float32 per frame],
    "messages": [...], "steps": [per captured step: dict of arrays], "masks": {...}}."""
    ref_main, particles, pressure_solve, voxelise_mesh = _import_reference(reference_root)
    record = {"steps": [], "masks": {}, "messages": []}
    originals = (voxelise_mesh.load_usdc_triangles, voxelise_mesh.build_static_masks,
                 particles.particle_to_grid, particles.grid_to_particle, pressure_solve.pressure_solve)

    def load_triangles(path):
        return np.ascontiguousarray(meshes[Path(path).name], dtype=np.float32)

    def build_static_masks(context, queue, kernel, simulation, grid_shape, delta):
        sources, obstacle = originals[1](context, queue, kernel, simulation, grid_shape, delta)
        record["masks"]["obstacle"] = _array(obstacle, np.uint8).reshape(grid_shape)
        for i, source in enumerate(sources):
            record["masks"][f"source{i}"] = _array(source["mask_device"], np.uint8).reshape(grid_shape)
        return sources, obstacle

    def particle_to_grid(*args):
        n, shape = int(args[11]), tuple(args[12])
        capture = len(record["steps"]) < capture_steps
        if capture:
            step = {"pos_in": _array(args[2], np.float32, 3 * n).reshape(n, 3),
                    "vel_in": _array(args[3], np.float32, 3 * n).reshape(n, 3)}
        result = originals[2](*args)
        if capture:
            cells = int(np.prod(shape))
            step.update(counts=_array(args[7], np.int32, cells).reshape(shape),
                        offsets=_array(args[8][0], np.int32, cells).reshape(shape),
                        pos_sorted=_array(result[0], np.float32, 3 * n).reshape(n, 3),
                        vel_sorted=_array(result[1], np.float32, 3 * n).reshape(n, 3),
                        p2g_u=_array(result[4][0], np.float32, cells).reshape(shape),
                        p2g_v=_array(result[4][1], np.float32, cells).reshape(shape),
                        p2g_w=_array(result[4][2], np.float32, cells).reshape(shape),
                        p2g_ff=_array(result[5], np.float32, cells).reshape(shape))
            record["steps"].append(step)
        return result

    def pressure_solve_hook(*args):
        shape = tuple(args[-1])
        cells = int(np.prod(shape))
        step = record["steps"][-1] if record["steps"] and "pressure" not in record["steps"][-1] else None
        if step is not None:
            u, v, w = args[4]
            step.update(pre_u=_array(u, np.float32, cells).reshape(shape),
                        pre_v=_array(v, np.float32, cells).reshape(shape),
                        pre_w=_array(w, np.float32, cells).reshape(shape),
                        ff=_array(args[5], np.float32, cells).reshape(shape),
                        pressure_in=_array(args[6], np.float32, cells).reshape(shape))
        result = originals[4](*args)
        if step is not None:
            step.update(rhs=_array(args[7], np.float32, cells).reshape(shape),
                        pressure=_array(result, np.float32, cells).reshape(shape))
        return result

    def grid_to_particle(*args):
        result = originals[3](*args)
        step = record["steps"][-1] if record["steps"] and "vel_g2p" not in record["steps"][-1] else None
        if step is not None:
            n, shape = int(args[6]), tuple(args[7])
            cells = int(np.prod(shape))
            step.update(vel_g2p=_array(result, np.float32, 3 * n).reshape(n, 3),
                        u=_array(args[4][0], np.float32, cells).reshape(shape),
                        v=_array(args[4][1], np.float32, cells).reshape(shape),
                        w=_array(args[4][2], np.float32, cells).reshape(shape))
        return result

    voxelise_mesh.load_usdc_triangles = load_triangles
    voxelise_mesh.build_static_masks = build_static_masks
    particles.particle_to_grid = particle_to_grid
    particles.grid_to_particle = grid_to_particle
    pressure_solve.pressure_solve = pressure_solve_hook
    with tempfile.TemporaryDirectory() as tmp:
        config = dict(config)
        simulation = dict(config["simulation"])
        simulation["output_path"] = str(Path(tmp) / "bake")
        config["simulation"] = simulation
        ref_main.set_message_callback(record["messages"].append)
        try:
            ref_main.main(config)
        finally:
            ref_main.clear_message_callback()
            (voxelise_mesh.load_usdc_triangles, voxelise_mesh.build_static_masks, particles.particle_to_grid,
             particles.grid_to_particle, pressure_solve.pressure_solve) = originals
        frames_dir = Path(tmp) / "bake" / "particles"
        record["frames"] = [np.fromfile(path, dtype=np.float32).reshape(-1, 3)
                            for path in sorted(frames_dir.glob("particles_*.bin"))]
    return record
