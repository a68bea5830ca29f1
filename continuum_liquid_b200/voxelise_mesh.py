"""Collider voxelisation stage (mirrors Solver/Kernel/voxelise_mesh.py).

The reference reads meshes from USD files through ``pxr`` (voxelise_mesh.py:74-100) and voxelises
them on the device. Here a geometry entry may carry its world-space triangles directly
(``{"triangles": float32 (T,3,3)}``); entries that name a USD file are read with ``pxr`` when it is
importable and rejected with a clear error otherwise. The device test is voxelise_mesh.cl.
"""

from __future__ import annotations

import numpy as np
import torch

from .backend import Backend


def world_triangles(triangles: np.ndarray, matrix_world) -> np.ndarray:
    """voxelise_mesh.py:104-109: ``tri @ M[:3,:3]^T + M[:3,3]`` in float32."""
    matrix = np.asarray(matrix_world, dtype=np.float32)
    flat = np.asarray(triangles, dtype=np.float32).reshape(-1, 3)
    world = flat @ matrix[:3, :3].T + matrix[:3, 3]
    return np.ascontiguousarray(world.reshape(-1, 3, 3), dtype=np.float32)


def _entry_triangles(entry, bake_path) -> np.ndarray:
    if "triangles" in entry:
        tris = np.ascontiguousarray(entry["triangles"], dtype=np.float32).reshape(-1, 3, 3)
        if "matrix_world" in entry:
            tris = world_triangles(tris, entry["matrix_world"])
        return tris
    try:
        from pxr import Usd, UsdGeom  # noqa: F401
    except ImportError as exc:  # pragma: no cover - pxr is not part of this environment
        raise RuntimeError(
            f"geometry entry {entry.get('object_name', '?')} names a USD file but pxr is not installed; "
            "pass world-space triangles in entry['triangles'] instead"
        ) from exc
    raise RuntimeError("USD mesh loading is outside this backend; pass entry['triangles']")  # pragma: no cover


def voxelise_triangles(kernels: Backend, queue, triangles, mask, grid_shape, delta, origin, cull: bool = True):
    """One voxelise_mesh launch (voxelise_mesh.py:120-134) OR-ing a mesh into ``mask``."""
    if isinstance(triangles, np.ndarray):
        triangles = torch.from_numpy(np.ascontiguousarray(triangles, dtype=np.float32)).to(kernels.device)
    count = int(triangles.numel() // 9)
    if count == 0:
        return mask
    nx, ny, nz = grid_shape
    kernels.call("clb_voxelise_mesh", triangles, mask, count, nx, ny, nz, float(np.float32(delta)),
                 float(np.float32(origin[0])), float(np.float32(origin[1])), float(np.float32(origin[2])),
                 1 if cull else 0, stream=queue)
    return mask


def voxelise_entries(context, queue, kernel, entries, bake_path, grid_shape, delta, origin):
    """voxelise_mesh.py:111-135: a zeroed uint8 mask with every entry's mesh OR-ed in.

    ``context`` and ``kernel`` are both the ``Backend`` here (the reference passes a cl.Context and
    the voxelise_mesh cl.Kernel).
    """
    kernels: Backend = kernel if isinstance(kernel, Backend) else context
    mask = torch.zeros(tuple(int(s) for s in grid_shape), dtype=torch.uint8, device=kernels.device)
    for entry in entries or ():
        tris = _entry_triangles(entry, bake_path)
        if not tris.size:
            continue
        voxelise_triangles(kernels, queue, tris, mask, grid_shape, delta, origin)
    return mask


def build_static_masks(context, queue, kernel, simulation, grid_shape, delta):
    """voxelise_mesh.py:138-163: source masks and the combined obstacle mask."""
    size = simulation["domain"]["size"]
    origin = (-0.5 * float(size["x"]), -0.5 * float(size["y"]), 0.0)
    bake_path = simulation.get("output_path", ".")
    sources = []
    for source in simulation.get("sources") or ():
        mask = voxelise_entries(context, queue, kernel, source.get("geometry_inputs"), bake_path, grid_shape, delta,
                                origin)
        sources.append({**source, "mask_device": mask})
    obstacles = [entry for obstacle in simulation.get("obstacles") or () for entry in
                 obstacle.get("geometry_inputs") or ()]
    obstacle_mask = voxelise_entries(context, queue, kernel, obstacles, bake_path, grid_shape, delta, origin)
    return sources, obstacle_mask


__all__ = ["world_triangles", "voxelise_triangles", "voxelise_entries", "build_static_masks"]
