"""Particle cache writer (mirrors Solver/Kernel/output.py; same on-disk format).

Layout: ``<dir>/particle_cache.json`` (metadata version 2) and ``<dir>/particles/particles_%06d.bin``
holding raw float32 (N, 3) positions. Frames are published atomically (written to ``.tmp`` then
renamed) so a reader polling the directory never sees a partial frame (output.py:46-53).

Device frames are copied into pinned host slots with an asynchronous copy on the solver's stream and
written by background threads; the solver thread does not wait for the copy (the writer waits on an
event recorded after it, and work queued later on the stream cannot overwrite the positions before
the copy has read them). A writer failure is re-raised on the solver thread at the next submit or at
close, as ``RuntimeError`` (output.py:91-97).
"""

from __future__ import annotations

import json
import queue as queue_module
import threading
from pathlib import Path
from typing import Any

import numpy as np
import torch

CACHE_FILENAME = "particle_cache.json"
FRAME_DIRECTORY = "particles"
FRAME_PATTERN = "particles_{frame:06d}.bin"
WRITER_COUNT = 2
PINNED_MEMORY_SLOTS = WRITER_COUNT + 1


def create_cache(directory, fps, start_frame, end_frame, particle_count=None) -> Path:
    """output.py:19-36: the frame directory and the version-2 metadata file."""
    directory = Path(directory)
    (directory / FRAME_DIRECTORY).mkdir(parents=True, exist_ok=True)
    metadata = {
        "version": 2,
        "fps": int(fps),
        "start_frame": int(start_frame),
        "end_frame": int(end_frame),
        "variable_particle_count": True,
        "dtype": "float32",
        "components": 3,
        "frame_directory": FRAME_DIRECTORY,
        "frame_pattern": FRAME_PATTERN,
    }
    (directory / CACHE_FILENAME).write_text(json.dumps(metadata, indent=2), encoding="utf-8")
    return directory


def write_particles(cache_directory, particles, frame) -> None:
    """output.py:39-53: write one frame to a temporary file, then rename it into place."""
    positions = np.ascontiguousarray(particles, dtype=np.float32)
    if positions.ndim != 2 or positions.shape[1] != 3:
        raise ValueError("Particle positions must have shape (N, 3)")
    path = Path(cache_directory) / FRAME_DIRECTORY / FRAME_PATTERN.format(frame=int(frame))
    tmp = path.with_suffix(path.suffix + ".tmp")
    try:
        positions.tofile(tmp)
        tmp.replace(path)
    finally:
        tmp.unlink(missing_ok=True)


def read_particles(cache_directory, frame) -> np.ndarray:
    """Inverse of write_particles (what Internal/Core/load_result.py:76-112 reads)."""
    path = Path(cache_directory) / FRAME_DIRECTORY / FRAME_PATTERN.format(frame=int(frame))
    return np.fromfile(path, dtype=np.float32).reshape(-1, 3)


class _Slot:
    __slots__ = ("host", "count", "frame", "ready")

    def __init__(self):
        self.host: torch.Tensor | None = None
        self.count = 0
        self.frame = 0
        self.ready: torch.cuda.Event | None = None  # recorded after the device-to-host copy

    def ensure(self, count: int) -> None:
        count = max(1, int(count))
        if self.host is None or self.host.shape[0] < count:
            pin = torch.cuda.is_available()
            self.host = torch.empty((count, 3), dtype=torch.float32, pin_memory=pin)


def _writer_loop(state: dict[str, Any]) -> None:
    while True:
        slot = state["write_queue"].get()
        try:
            if slot is None:
                return
            if slot.ready is not None:
                slot.ready.synchronize()
                slot.ready = None
            write_particles(state["cache_directory"], slot.host[: slot.count].numpy(), slot.frame)
        except BaseException as exc:  # noqa: BLE001 - collected and re-raised on the solver thread
            with state["error_lock"]:
                state["errors"].append(exc)
        finally:
            if slot is not None:
                state["free_slots"].put(slot)
            state["write_queue"].task_done()


def create_output(cache_directory) -> dict[str, Any]:
    """output.py:110-143: pinned slots and writer threads."""
    state: dict[str, Any] = {
        "cache_directory": Path(cache_directory),
        "free_slots": queue_module.Queue(PINNED_MEMORY_SLOTS),
        "write_queue": queue_module.Queue(PINNED_MEMORY_SLOTS),
        "threads": [],
        "errors": [],
        "error_lock": threading.Lock(),
        "closed": False,
    }
    for _ in range(PINNED_MEMORY_SLOTS):
        state["free_slots"].put(_Slot())
    for index in range(WRITER_COUNT):
        thread = threading.Thread(target=_writer_loop, args=(state,), name=f"ContinuumParticleWriter-{index + 1}",
                                  daemon=True)
        thread.start()
        state["threads"].append(thread)
    return state


def _raise_writer_error(state: dict[str, Any]) -> None:
    with state["error_lock"]:
        if state["errors"]:
            raise RuntimeError("Asynchronous particle writer failed") from state["errors"][0]


def _acquire_slot(state: dict[str, Any], count: int, frame: int) -> _Slot:
    _raise_writer_error(state)
    if state["closed"]:
        raise RuntimeError("Particle output is already closed")
    slot: _Slot = state["free_slots"].get()
    slot.ensure(count)
    slot.count = int(count)
    slot.frame = int(frame)
    return slot


def submit_host(state: dict[str, Any], particles, frame: int) -> None:
    """output.py:158-166: queue a host array for writing."""
    positions = np.ascontiguousarray(particles, dtype=np.float32)
    if positions.ndim != 2 or positions.shape[1] != 3:
        raise ValueError("Particle positions must have shape (N, 3)")
    slot = _acquire_slot(state, len(positions), frame)
    if len(positions):
        slot.host[: len(positions)].copy_(torch.from_numpy(positions))
    state["write_queue"].put(slot)


def submit_output(state: dict[str, Any], *, particles: torch.Tensor, particle_count: int, frame: int,
                  queue=None) -> None:
    """output.py:169-186: copy the first ``particle_count`` device positions into a pinned slot
    (asynchronous copy on the current stream) and queue it for writing; the writer thread waits for
    the copy, the caller does not."""
    slot = _acquire_slot(state, particle_count, frame)
    if particle_count:
        slot.host[:particle_count].copy_(particles[:particle_count], non_blocking=True)
        slot.ready = torch.cuda.Event()
        slot.ready.record()
    state["write_queue"].put(slot)


def close_output(state: dict[str, Any]) -> None:
    """output.py:189-199: drain the queue, stop the threads, re-raise a writer failure."""
    if state["closed"]:
        return
    state["closed"] = True
    state["write_queue"].join()
    for _ in state["threads"]:
        state["write_queue"].put(None)
    for thread in state["threads"]:
        thread.join()
    _raise_writer_error(state)
