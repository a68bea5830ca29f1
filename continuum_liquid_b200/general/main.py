"""Solver entry point and runtime message channel (mirrors Solver/General/main.py).

The add-on's bake operator calls ``main(config)`` on a worker thread after registering a message
callback; the solver reports progress through ``emit_message``. Backend strings "CPU" and "GPU" are
both accepted as in the reference (main.py:41-46) and both run on the B200 backend: there is no CPU
implementation behind this entry point. Any other backend raises ``ValueError`` (main.py:48).
"""

from __future__ import annotations

import threading
from time import perf_counter
from typing import Any, Callable

MessageCallback = Callable[[dict[str, Any]], None]

_message_callback: MessageCallback | None = None
_message_callback_lock = threading.Lock()


def set_message_callback(callback: MessageCallback | None) -> None:
    """main.py:13-17."""
    global _message_callback
    with _message_callback_lock:
        _message_callback = callback


def clear_message_callback() -> None:
    """main.py:20-24."""
    global _message_callback
    with _message_callback_lock:
        _message_callback = None


def emit_message(message: dict[str, Any]) -> None:
    """main.py:27-32: forward a runtime message to the active caller (outside the lock)."""
    with _message_callback_lock:
        callback = _message_callback
    if callback is not None:
        callback(message)


def main(config: dict[str, Any]) -> None:
    """main.py:35-52: select the configured backend and run the solver."""
    total_start_time = perf_counter()
    try:
        simulation_config = config.get("simulation") or {}
        settings = simulation_config.get("settings") or {}
        solver_backend = str(settings.get("solver_backend", "CPU")).strip().upper()
        if solver_backend in {"CPU", "GPU"}:
            from .. import solver as solver_kernel_module

            return solver_kernel_module.solver(config)
        raise ValueError(f"Unsupported solver backend: {solver_backend}")
    finally:
        total_runtime = perf_counter() - total_start_time
        print(f"Bake runtime: {total_runtime:.3f} s")
        print("################################################################")
