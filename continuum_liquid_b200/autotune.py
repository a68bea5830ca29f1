"""Per-level choice of the red-black sweep implementation, by measurement.

Every sweep kind of clb_mg_hierarchy.sweep gives identical values; which one is fastest depends on
the level's size (large levels are bandwidth- or issue-bound, small ones latency-bound). The tuner
times each candidate kind on the live operator of each level with CUDA events and keeps the
fastest. Results are cached per process, keyed by device name and level shapes.
"""

from __future__ import annotations

import torch

KINDS = {
    1: "two colour launches, 16-byte row vectors",
    2: "fused iteration, 8x8x32 tiles",
    3: "fused iteration, 4x4x32 tiles",
    4: "two colour launches, one thread per cell",
    5: "fused pairs of iterations, 8x8x32 tiles",
    6: "fused pairs of iterations, 4x4x32 tiles",
}

_cache: dict[tuple, dict[int, int]] = {}


def _time_smooth(h, level, x, rhs, iterations, repeats) -> float:
    h.smooth(level, 1, x, rhs)  # warm-up
    best = float("inf")
    for _ in range(repeats):
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        h.smooth(level, iterations, x, rhs)
        end.record()
        end.synchronize()
        best = min(best, start.elapsed_time(end) / iterations)
    return best


def tune_hierarchy(h, x, rhs, iterations: int = 4, repeats: int = 3) -> dict[int, int]:
    """Pick a sweep kind for every level that runs red-black sweeps (``x``/``rhs``: level-0 buffers
    the sweeps may overwrite). Returns {level: kind} and writes it into the hierarchy."""
    key = (torch.cuda.get_device_name(h.kernels.device), tuple(h.shapes), getattr(h, "fp16_level", 0))
    choice = _cache.get(key)
    if choice is None:
        choice = {}
        timings = {}
        for level in range(h.levels - 1):
            # FP32 coarse levels have no two-iteration 8x8x32 tile (kind 5 runs as 6 there)
            fused = ([2, 3, 5, 6] if level == 0 or h.is_fp16(level) else [2, 3, 6]) if h.alt[level] is not None else []
            candidates = ([4] if h.is_fp16(level) else [1, 4]) + fused
            times = {}
            for kind in candidates:
                h.set_sweep(level, kind)
                times[kind] = _time_smooth(h, level, x if level == 0 else None, rhs if level == 0 else None,
                                           iterations, repeats)
            choice[level] = min(times, key=times.get)
            timings[level] = times
        _cache[key] = choice
        h.tuning = timings
    for level, kind in choice.items():
        h.set_sweep(level, kind)
    return choice
