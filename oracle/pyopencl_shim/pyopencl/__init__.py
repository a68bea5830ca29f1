"""A stand-in for pyopencl that runs OpenCL programs on the host CPU. Test infrastructure only.

It implements the part of pyopencl's API that the reference's host code (Solver/Kernel/*.py) calls:
one platform with one device, contexts, in-order queues, buffers backed by host memory, copies,
fills and maps, and programs. `Program.build` hands the program text and build options to
`oracle/ref_build.py`, which rewrites the OpenCL C into C++ over `oracle/clshim.h` and compiles it
into oracle/_ref/; a kernel call runs the compiled kernel over the NDRange on the calling thread
(oracle/clshim_runtime.cpp). Every command completes before the call returns, so events are
already complete and `finish()` has nothing to wait for.

Put this directory first on sys.path to import it as `pyopencl`.
"""

from __future__ import annotations

import ctypes
import itertools
from pathlib import Path

import numpy as np

_ORACLE_DIR = Path(__file__).resolve().parents[2]


def _load_ref_build():
    """oracle/ref_build.py, loaded by path (putting oracle/ on sys.path would shadow the package)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("clb_oracle_ref_build", _ORACLE_DIR / "ref_build.py")
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


ref_build = _load_ref_build()

# Kernels whose work-groups write disjoint memory (their own cell, particle or group) and use no
# atomics, so running their groups on several threads cannot change any result. Every other kernel
# runs its work-groups one after another in order (the Gauss-Seidel sweep updates in place, the
# counting sort hands out slots with atomic_inc in work-item order, the boundary kernels read cells
# that other work-items write).
PARALLEL_KERNELS = {"voxelise_mesh", "particle_to_grid_gather", "grid_to_particle", "advect_particles"}
THREADS = max(1, int(__import__("os").environ.get("CLSHIM_THREADS", __import__("os").cpu_count() or 1)))

VERSION = (2026, 1)
VERSION_TEXT = "host shim"
_ids = itertools.count(1)


class CompilerWarning(UserWarning):
    pass


class Error(RuntimeError):
    pass


class LogicError(Error):
    pass


class RuntimeError(Error):  # noqa: A001  (pyopencl's own name)
    pass


class mem_flags:  # noqa: N801
    READ_WRITE = 1 << 0
    WRITE_ONLY = 1 << 1
    READ_ONLY = 1 << 2
    USE_HOST_PTR = 1 << 3
    ALLOC_HOST_PTR = 1 << 4
    COPY_HOST_PTR = 1 << 5


class map_flags:  # noqa: N801
    READ = 1 << 0
    WRITE = 1 << 1
    WRITE_INVALIDATE_REGION = 1 << 2


class device_type:  # noqa: N801
    DEFAULT = 1 << 0
    CPU = 1 << 1
    GPU = 1 << 2
    ACCELERATOR = 1 << 3
    ALL = 0xFFFFFFFF


class kernel_work_group_info:  # noqa: N801
    WORK_GROUP_SIZE = 0x11B0
    COMPILE_WORK_GROUP_SIZE = 0x11B1
    LOCAL_MEM_SIZE = 0x11B2
    PREFERRED_WORK_GROUP_SIZE_MULTIPLE = 0x11B3
    PRIVATE_MEM_SIZE = 0x11B4


class Device:
    """One device with GPU-like limits (work-groups up to 1024 work-items, 48 KiB local memory)."""

    def __init__(self, kind: int):
        self.type = kind
        self.name = "host shim device"
        self.vendor = "oracle"
        self.max_work_group_size = 1024
        self.max_work_item_sizes = [1024, 1024, 64]
        self.local_mem_size = 48 * 1024
        self.max_compute_units = 148
        self.int_ptr = next(_ids)


class Platform:
    def __init__(self):
        self.name = "host shim platform"
        self._devices = {device_type.GPU: Device(device_type.GPU), device_type.CPU: Device(device_type.CPU)}

    def get_devices(self, device_type=None):  # noqa: A002  (pyopencl's keyword)
        if device_type is None or device_type == 0xFFFFFFFF:
            return list(self._devices.values())
        return [d for kind, d in self._devices.items() if kind & device_type]


_PLATFORM = Platform()


def get_platforms():
    return [_PLATFORM]


class Context:
    def __init__(self, devices=None, properties=None, dev_type=None):
        self.devices = list(devices or _PLATFORM.get_devices())
        self.int_ptr = next(_ids)


class Event:
    def wait(self):
        return None


class CommandQueue:
    def __init__(self, context, device=None, properties=None):
        self.context = context
        self.device = device or context.devices[0]
        self.int_ptr = next(_ids)

    def finish(self):
        return None

    def flush(self):
        return None


class Buffer:
    """Device memory as a 64-byte aligned host byte array."""

    def __init__(self, context, flags, size=0, hostbuf=None):
        if hostbuf is not None:
            host = np.ascontiguousarray(hostbuf)
            size = size or host.nbytes
        if size <= 0:
            raise LogicError("Buffer size must be positive")
        self.context = context
        self.flags = flags
        self.size = int(size)
        raw = np.zeros(self.size + 64, dtype=np.uint8)
        start = (-raw.ctypes.data) % 64
        self._raw = raw
        self.bytes = raw[start : start + self.size]
        self.int_ptr = self.bytes.ctypes.data
        if hostbuf is not None and flags & (mem_flags.COPY_HOST_PTR | mem_flags.USE_HOST_PTR):
            data = host.reshape(-1).view(np.uint8)
            self.bytes[: data.nbytes] = data


class LocalMemory:
    def __init__(self, size):
        self.size = int(size)


def _host_bytes(array) -> np.ndarray:
    array = np.asarray(array)
    if not array.flags.c_contiguous:
        raise LogicError("host arrays must be contiguous")
    return array.reshape(-1).view(np.uint8)


def enqueue_copy(queue, dest, src, is_blocking=True, wait_for=None, byte_count=None, src_offset=0,
                 dst_offset=0, device_offset=0, **_):
    if isinstance(dest, Buffer) and isinstance(src, Buffer):
        count = src.size - src_offset if byte_count is None else int(byte_count)
        dest.bytes[dst_offset : dst_offset + count] = src.bytes[src_offset : src_offset + count]
    elif isinstance(dest, Buffer):
        data = _host_bytes(src)
        count = data.nbytes if byte_count is None else int(byte_count)
        off = device_offset or dst_offset
        dest.bytes[off : off + count] = data[:count]
    elif isinstance(src, Buffer):
        out = _host_bytes(dest)
        count = out.nbytes if byte_count is None else int(byte_count)
        off = device_offset or src_offset
        out[:count] = src.bytes[off : off + count]
    else:
        raise LogicError("enqueue_copy needs a Buffer on at least one side")
    return Event()


def enqueue_fill_buffer(queue, mem, pattern, offset, size, wait_for=None):
    pattern = np.ascontiguousarray(pattern).reshape(-1).view(np.uint8)
    size = int(size)
    repeats = size // pattern.nbytes
    mem.bytes[offset : offset + repeats * pattern.nbytes] = np.tile(pattern, repeats)
    return Event()


def enqueue_map_buffer(queue, buf, flags, offset, shape, dtype, order="C", strides=None, wait_for=None,
                       is_blocking=True):
    dtype = np.dtype(dtype)
    count = int(np.prod(shape)) * dtype.itemsize
    array = buf.bytes[offset : offset + count].view(dtype).reshape(shape)
    return array, Event()


def enqueue_barrier(queue, wait_for=None):
    return Event()


def enqueue_marker(queue, wait_for=None):
    return Event()


def wait_for_events(events):
    return None


# ---- programs and kernels -------------------------------------------------------------------------
class _Library:
    def __init__(self, path: Path):
        self.dll = ctypes.CDLL(str(path))
        self.dll.clshim_kernel_name.restype = ctypes.c_char_p
        self.dll.clshim_last_error.restype = ctypes.c_char_p
        self.dll.clshim_launch.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t),
                                           ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_void_p),
                                           ctypes.POINTER(ctypes.c_longlong), ctypes.c_int, ctypes.c_int]
        self.kernels = {self.dll.clshim_kernel_name(i).decode(): (i, self.dll.clshim_kernel_arity(i))
                        for i in range(self.dll.clshim_kernel_count())}


class Kernel:
    def __init__(self, library: _Library, name: str):
        self._library = library
        self.function_name = name
        self._index, self.num_args = library.kernels[name]
        self._args = None

    def get_work_group_info(self, param, device):
        if param == kernel_work_group_info.WORK_GROUP_SIZE:
            return device.max_work_group_size
        if param == kernel_work_group_info.PREFERRED_WORK_GROUP_SIZE_MULTIPLE:
            return 32
        return 0

    def set_args(self, *args):
        self._args = args

    def __call__(self, queue, global_size, local_size, *args, wait_for=None, g_times_l=False):
        if not args and self._args is not None:
            args = self._args
        if len(args) != self.num_args:
            raise LogicError(f"{self.function_name}: {self.num_args} arguments expected, {len(args)} given")
        dims = len(global_size)
        gsize = (ctypes.c_size_t * 3)(*[int(g) for g in global_size], *([1] * (3 - dims)))
        lsize = None
        if local_size is not None:
            lsize = (ctypes.c_size_t * 3)(*[int(g) for g in local_size], *([1] * (3 - dims)))
            if g_times_l:
                for d in range(dims):
                    gsize[d] *= lsize[d]
        slots = (ctypes.c_uint64 * max(1, len(args)))()
        local_bytes = (ctypes.c_longlong * max(1, len(args)))()
        for i, arg in enumerate(args):
            if isinstance(arg, Buffer):
                slots[i] = arg.int_ptr
            elif isinstance(arg, LocalMemory):
                local_bytes[i] = arg.size
            elif arg is None:
                slots[i] = 0
            elif isinstance(arg, np.generic):
                raw = np.zeros(8, dtype=np.uint8)
                raw[: arg.nbytes] = np.frombuffer(arg.tobytes(), dtype=np.uint8)
                slots[i] = int(raw.view(np.uint64)[0])
            else:
                raise LogicError(f"{self.function_name}: argument {i} must be a Buffer, LocalMemory or a numpy "
                                 f"scalar, got {type(arg).__name__}")
        base = ctypes.addressof(slots)
        argv = (ctypes.c_void_p * max(1, len(args)))(*[base + 8 * i for i in range(len(args))])
        threads = THREADS if self.function_name in PARALLEL_KERNELS else 1
        status = self._library.dll.clshim_launch(self._index, dims, gsize, lsize, argv, local_bytes, len(args),
                                                 threads)
        if status != 0:
            raise LogicError(self._library.dll.clshim_last_error().decode())
        return Event()


class Program:
    def __init__(self, context, source):
        self.context = context
        self.source = source
        self._library = None

    def build(self, options=None, devices=None, cache_dir=None):
        if isinstance(options, str):
            options = [options]
        names = ref_build._KERNEL.findall(self.source)
        path = ref_build.build_program(self.source, options or (), names[0] if names else "program")
        self._library = _Library(path)
        return self

    def all_kernels(self):
        return [Kernel(self._library, name) for name in self._library.kernels]

    def __getattr__(self, name):
        library = self.__dict__.get("_library")
        if library is not None and name in library.kernels:
            return Kernel(library, name)
        raise AttributeError(name)
