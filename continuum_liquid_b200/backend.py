"""ctypes binding of libclb200.so (include/clb200.h).

``Backend`` replaces the reference's OpenCL context, queue and kernel dictionaries
(Solver/Kernel/helper.py:22-69, solver.py:29-82): it loads the CUDA library, selects the device and
exposes every C entry point as a method taking torch tensors. A non-zero status from the library
becomes ``RuntimeError(clb_last_error())``, the exception type the reference raises for device and
runtime failures (helper.py:55,64; output.py:94-96).

There is no CPU path: if the library is missing or no B200 is visible, constructing a Backend
raises.
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path
from typing import Any

import torch

from . import build as _build

LIBRARY_PATH = _build.LIBRARY
MG_MAX_LEVELS = 16
SCAN_TILE = 4096  # elements per scan tile (SCAN_THREADS * SCAN_ITEMS in csrc/binning.cuh)

P, I, L, F, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_float, ctypes.c_double
U = ctypes.c_uint64

# name -> argument types (every entry point returns int status unless listed in _RESTYPES)
SIGNATURES: dict[str, list[Any]] = {
    "clb_init": [I],
    "clb_last_error": [],
    "clb_device_error": [P],
    "clb_abi_version": [],
    "clb_launch_count": [],
    "clb_count_particles_per_cell": [P, P, P, P, L, F, I, I, I, P],
    "clb_scan_scratch_bytes": [L],
    "clb_exclusive_prefix_sum": [P, P, P, L, P, L, P],
    "clb_exclusive_prefix_sum_static": [P, P, P, L, P],
    "clb_sort_particles": [P, P, P, P, P, P, P, P, P, P, L, P],
    "clb_particle_to_grid_gather": [P, P, P, P, P, P, P, P, F, F, I, I, I, P],
    "clb_particle_to_grid": [P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, L, L, F, F, I, I, I, P],
    "clb_particle_to_grid_gather_tiled": [P, P, P, P, P, P, P, P, F, F, I, I, I, P],
    "clb_particle_to_grid_tiled": [P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, L, L, F, F, I, I, I, P],
    "clb_grid_to_particle": [P, P, P, P, P, P, P, P, L, F, I, I, I, F, P],
    "clb_advect_particles": [P, P, L, F, P],
    "clb_particle_domain_bc": [P, P, L, F, F, F, F, P],
    "clb_particle_obstacle_bc": [P, P, P, P, L, F, I, I, I, P],
    "clb_particle_update": [P, P, P, P, P, P, P, P, P, P, L, F, I, I, I, F, F, F, F, F, F, P],
    "clb_particle_update_moving": [P, P, P, P, P, P, P, P, P, P, L, F, I, I, I, F, F, F, F, F, F, P, P],
    "clb_particle_update_tiled": [P, P, P, P, P, P, P, P, P, P, P, P, L, F, I, I, I, F, F, F, F, F, F, P, P],
    "clb_particle_obstacle_bc_moving": [P, P, P, P, L, F, I, I, I, P, P],
    "clb_grid_obstacle_bc_moving": [P, P, P, P, P, I, I, I, P, F, P],
    "clb_update_velocity": [P, P, P, P, P, P, P, F, F, F, F, F, F, F, F, F, F, I, I, I, P],
    "clb_grid_domain_bc": [P, P, P, I, I, I, P],
    "clb_grid_obstacle_bc": [P, P, P, P, P, I, I, I, P],
    "clb_pressure_rhs": [P, P, P, P, P, F, F, I, I, I, P],
    "clb_pressure_correction": [P, P, P, P, F, F, I, I, I, P],
    "clb_neumann_domain_bc": [P, I, I, I, P],
    "clb_pressure_correction_f64": [P, P, P, P, F, F, I, I, I, P],
    "clb_neumann_domain_bc_f64": [P, I, I, I, P],
    "clb_mg_pack_finest": [P, P, P, P, P, P, P, I, I, I, P],
    "clb_mg_unpack_finest": [P, P, P, P, P, I, I, I, P],
    "clb_mg_pack_level": [P, P, P, P, P, P, P, I, I, I, P],
    "clb_mg_unpack_level": [P, P, P, P, P, P, P, I, I, I, P],
    "clb_mg_smooth_level": [P, P, P, P, F, I, I, I, I, P],
    "clb_mg_coarse_solve_level": [P, P, P, P, F, I, I, I, I, P],
    "clb_mg_rhs_operator": [P, P, P, P, P, P, F, F, I, I, I, P],
    "clb_source_cell_counts": [P, L, F, I, I, I, P, P],
    "clb_source_keep": [P, L, F, I, I, I, P, P, P],
    "clb_source_compact": [P, P, P, P, L, P, P, P],
    "clb_source_missing": [P, P, P, I, L, P, P],
    "clb_source_spawn": [P, P, I, I, I, D, F, F, F, U, U, U, U, P, P, P],
    "clb_batch_particle_to_grid": [P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, L, F, P],
    "clb_batch_update_velocity": [P, P, P, P, P, P, P, P, F, F, F, F, F, F, F, F, F, P],
    "clb_batch_grid_domain_bc": [P, P, P, P, P],
    "clb_batch_grid_obstacle_bc": [P, P, P, P, P, P, P],
    "clb_batch_rhs_operator": [P, P, P, P, P, P, P],
    "clb_batch_w_cycle": [P, P, P, I, I, I, P],
    "clb_batch_residual_norms": [P, P, I, P, P, P, P, P],
    "clb_batch_ir_init": [P, P, P, P],
    "clb_batch_ir_store": [P, P, P, P],
    "clb_batch_fcg_dots": [P, P, P, P, P, P, P],
    "clb_batch_fcg_step": [P, P, P, P, P, P, P, P, P, P, P, P],
    "clb_batch_pressure_correction": [P, P, P, P, P, I, P],
    "clb_batch_neumann_domain_bc": [P, P, P],
    "clb_batch_particle_update": [P, P, P, P, P, P, P, P, P, P, F, F, P],
    "clb_mg_build_coarse": [P, P],
    "clb_mg_w_cycle": [P, P, P, I, I, I, P],
    "clb_mg_smooth": [P, I, P, P, I, P],
    "clb_mg_level0_iteration": [P, P, P, P, I, P],
    "clb_solve_loop_create": [P, P, P, P, P, P, P, P, P, P, P, P, I, I, I, I, D, I, P, P, I, P],
    "clb_solve_loop_launch": [P, P, P],
    "clb_solve_loop_launches": [P],
    "clb_solve_loop_destroy": [P],
    "clb_mg_set_option": [I, I],
    "clb_mg_residual_partials": [L],
    "clb_mg_tile_capacity": [I, I, I, I],
    "clb_mg_fused_tile_capacity": [I, I, I],
    "clb_mg_cluster_list_capacity": [P],
    "clb_mg_residual_norms": [P, I, P, P, F, I, I, I, P, P, P, P],
    "clb_mg_ir_init": [P, P, P, I, I, I, P],
    "clb_mg_ir_step": [P, P, P, P, P, F, I, I, I, P, P, P, P],
    "clb_mg_fcg_dots": [P, P, P, P, F, I, I, I, P, P, P],
    "clb_mg_fcg_step": [P, P, P, P, P, P, P, P, F, I, I, I, P, P, P, P],
    "clb_mg_ir_update": [P, P, L, P],
    "clb_mg_ir_store": [P, P, L, P],
    "clb_tc_test_gemm": [P, P, P, I, I, I, I, P],
    "clb_conv3d_arrange_weights": [P, P, P, I, I, I, I, P],
    "clb_conv3d_forward": [P, P, P, P, I, I, I, I, I, I, I, I, P],
    "clb_conv3d_dgrad": [P, P, P, P, I, I, I, I, I, I, I, P],
    "clb_conv3d_wgrad": [P, P, P, I, I, I, I, I, I, I, P],
    "clb_unet_avgpool2": [P, P, I, I, I, I, I, P],
    "clb_unet_avgpool2_backward": [P, P, P, I, I, I, I, I, P],
    "clb_unet_upsample_concat": [P, P, P, I, I, I, I, I, I, P],
    "clb_unet_upsample_concat_backward": [P, P, P, I, I, I, I, I, I, P],
    "clb_unet_head_forward": [P, P, P, P, I, I, P],
    "clb_unet_head_backward": [P, P, P, P, P, P, I, I, P],
    "clb_unet_bias_grad": [P, P, I, I, P],
    "clb_adam_step": [P, P, P, P, L, F, F, F, F, I, P],
    "clb_unet_pack_input": [P, P, P, P, F, F, I, I, I, I, I, I, P, I, I, I, I, P],
    "clb_unet_pack_target": [P, P, P, F, I, I, I, I, I, I, P, P, I, I, I, I, P],
    "clb_unet_unpack_output": [P, P, P, F, P, I, I, I, I, I, I, P],
    "clb_unet_mse": [P, P, P, P, P, L, F, P],
    "clb_voxelise_mesh": [P, P, I, I, I, I, F, F, F, F, I, P],
    "clb_voxelise_direction": [P],
}
_RESTYPES = {
    "clb_last_error": ctypes.c_char_p,
    "clb_scan_scratch_bytes": ctypes.c_int64,
    "clb_launch_count": ctypes.c_int64,
    "clb_mg_tile_capacity": ctypes.c_int64,
    "clb_mg_fused_tile_capacity": ctypes.c_int64,
    "clb_mg_cluster_list_capacity": ctypes.c_int64,
}


class MGHierarchy(ctypes.Structure):
    """Mirror of clb_mg_hierarchy (include/clb200.h)."""

    _fields_ = [
        ("levels", ctypes.c_int32),
        ("shape", (ctypes.c_int32 * 3) * MG_MAX_LEVELS),
        ("delta", ctypes.c_float),
        ("fp16_level", ctypes.c_int32),
        ("op0", ctypes.c_void_p),
        ("p", ctypes.c_void_p * MG_MAX_LEVELS),
        ("b", ctypes.c_void_p * MG_MAX_LEVELS),
        ("mask", ctypes.c_void_p * MG_MAX_LEVELS),
        ("op", ctypes.c_void_p * MG_MAX_LEVELS),
        ("alt", ctypes.c_void_p * MG_MAX_LEVELS),
        ("sweep", ctypes.c_int32 * MG_MAX_LEVELS),
        ("fp16_scale", ctypes.c_void_p),
        ("rhs_norms", ctypes.c_void_p),
        ("fp16_inexact", ctypes.c_void_p),
        ("tiles", ctypes.c_void_p * MG_MAX_LEVELS),
        ("tile_counts", ctypes.c_void_p),
        ("zero_outside", ctypes.c_int32),
        ("fused_tiles", ctypes.c_void_p),
        ("fused_tile_count", ctypes.c_void_p),
        ("cluster_lists", ctypes.c_void_p),
        ("prolong_scale", ctypes.c_float),
        ("coarse_smoothing", ctypes.c_int32),
        ("coarse_pre_smooth", ctypes.c_int32),
        ("coarse_post_smooth", ctypes.c_int32),
    ]


BATCH_MAX_SCENES = 64


class BatchScene(ctypes.Structure):
    """Mirror of clb_batch_scene (include/clb200.h)."""

    _fields_ = [
        ("levels", ctypes.c_int32),
        ("bottom", ctypes.c_int32),
        ("shape", (ctypes.c_int32 * 3) * MG_MAX_LEVELS),
        ("base", ctypes.c_int64 * MG_MAX_LEVELS),
        ("particle_base", ctypes.c_int64),
        ("particles", ctypes.c_int64),
        ("delta", ctypes.c_float),
        ("inv_dx", ctypes.c_float),
        ("inv_dx2", ctypes.c_float),
        ("rho_over_dt", ctypes.c_float),
        ("dt_over_rho", ctypes.c_float),
        ("lower", ctypes.c_float),
        ("upper", ctypes.c_float * 3),
        ("pad", ctypes.c_int32),
    ]


class BatchList(ctypes.Structure):
    """Mirror of clb_batch_list."""

    _fields_ = [
        ("scene", ctypes.c_void_p),
        ("start", ctypes.c_void_p),
        ("count", ctypes.c_int32),
        ("pad", ctypes.c_int32),
        ("total", ctypes.c_int64),
    ]


class Batch(ctypes.Structure):
    """Mirror of clb_batch."""

    _fields_ = [
        ("scenes", ctypes.c_int32),
        ("levels", ctypes.c_int32),
        ("geom", ctypes.c_void_p),
        ("geom_host", ctypes.c_void_p),
        ("particles", BatchList),
        ("cells", BatchList * MG_MAX_LEVELS),
        ("recurse", BatchList * MG_MAX_LEVELS),
        ("recurse_coarse", BatchList * MG_MAX_LEVELS),
        ("bottom", BatchList * MG_MAX_LEVELS),
        ("coarse", BatchList * MG_MAX_LEVELS),
        ("colour0", BatchList),
        ("sweep0", ctypes.c_int32),
        ("vec0", ctypes.c_int32),
        ("reduce_blocks", ctypes.c_int32),
        ("bottom_ka", ctypes.c_int32),
        ("bottom_kb", ctypes.c_int32),
        ("p2g_tiled", ctypes.c_int32),
        ("bottom_smem", ctypes.c_int64),
        ("op0", ctypes.c_void_p),
        ("p", ctypes.c_void_p * MG_MAX_LEVELS),
        ("b", ctypes.c_void_p * MG_MAX_LEVELS),
        ("mask", ctypes.c_void_p * MG_MAX_LEVELS),
        ("op", ctypes.c_void_p * MG_MAX_LEVELS),
        ("prolong_scale", ctypes.c_float),
        ("coarse_smoothing", ctypes.c_int32),
        ("coarse_pre_smooth", ctypes.c_int32),
        ("coarse_post_smooth", ctypes.c_int32),
    ]


def load_library(path: Path | str = LIBRARY_PATH) -> ctypes.CDLL:
    """Load libclb200.so and declare every entry point's signature (no device work)."""
    path = Path(path)
    if not path.exists():
        raise RuntimeError(
            f"{path.name} is not built; run `python -m continuum_liquid_b200.build` (needs nvcc) before use"
        )
    lib = ctypes.CDLL(str(path))
    for name, argtypes in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = _RESTYPES.get(name, ctypes.c_int)
    return lib


def ptr(t: torch.Tensor | None) -> int | None:
    """Device address of a contiguous tensor (None -> NULL)."""
    if t is None:
        return None
    if not t.is_contiguous():
        raise ValueError("tensors passed to the CUDA backend must be contiguous")
    return t.data_ptr()


class Backend:
    """Loaded CUDA library bound to one device; methods enqueue on the given (or current) stream."""

    _lock = threading.Lock()
    _lib: ctypes.CDLL | None = None

    def __init__(self, device: int | torch.device = 0):
        if not torch.cuda.is_available():
            raise RuntimeError("No CUDA device found: the Continuum Liquid B200 backend needs a B200 GPU")
        self.device = torch.device("cuda", device if isinstance(device, int) else device.index or 0)
        with Backend._lock:
            if Backend._lib is None:
                Backend._lib = load_library()
        self.lib = Backend._lib
        torch.cuda.set_device(self.device)
        self._check(self.lib.clb_init(self.device.index), "clb_init")
        direction = (ctypes.c_float * 3)()
        self._check(self.lib.clb_voxelise_direction(direction), "clb_voxelise_direction")
        self.voxelise_direction = tuple(float(x) for x in direction)

    # -- plumbing -----------------------------------------------------------------------------
    def _check(self, status: int, name: str) -> None:
        if status != 0:
            message = (self.lib.clb_last_error() or b"").decode(errors="replace")
            raise RuntimeError(f"{name} failed: {message}")

    def stream_handle(self, stream: torch.cuda.Stream | None = None) -> int:
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        return s.cuda_stream

    def call(self, name: str, *args: Any, stream: torch.cuda.Stream | None = None) -> None:
        """Invoke entry point `name`; tensors are passed as device pointers, the stream last."""
        converted = [ptr(a) if isinstance(a, torch.Tensor) or a is None else a for a in args]
        self._check(getattr(self.lib, name)(*converted, self.stream_handle(stream)), name)

    def device_error(self) -> int:
        code = ctypes.c_uint32(0)
        self._check(self.lib.clb_device_error(ctypes.byref(code)), "clb_device_error")
        return int(code.value)

    def scan_scratch_bytes(self, count: int) -> int:
        return int(self.lib.clb_scan_scratch_bytes(count))

    @staticmethod
    def scan_scratch_bytes_static(count: int) -> int:
        """Same value as clb_scan_scratch_bytes without loading the library: a 16-byte ticket
        header plus one 8-byte look-back status word per 4096-element tile."""
        tiles = (int(count) + SCAN_TILE - 1) // SCAN_TILE
        return 16 + 8 * max(tiles, 1)

    def launch_count(self) -> int:
        """Kernels launched directly by the library so far (graph replays excluded)."""
        return int(self.lib.clb_launch_count())

    def residual_partials(self, cells: int) -> int:
        return int(self.lib.clb_mg_residual_partials(cells))

    def call_batch(self, name: str, batch: "Batch", *args: Any, stream=None) -> None:
        """Call a clb_batch_* entry point (the batch struct is passed by pointer)."""
        self.call_hierarchy(name, batch, *args, stream=stream)

    def call_hierarchy(self, name: str, hierarchy: MGHierarchy, *args: Any, stream=None) -> None:
        converted = [ptr(a) if isinstance(a, torch.Tensor) or a is None else a for a in args]
        status = getattr(self.lib, name)(ctypes.byref(hierarchy), *converted, self.stream_handle(stream))
        self._check(status, name)


_default: Backend | None = None


def default_backend() -> Backend:
    """Process-wide backend on cuda:0 (the reference serves compute_devices[0], helper.py:62-69)."""
    global _default
    if _default is None:
        _default = Backend(0)
    return _default
