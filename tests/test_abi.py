"""The C ABI library loads and exports every symbol include/clb200.h declares (no device work)."""

import ctypes
import re
from pathlib import Path

from continuum_liquid_b200 import backend, build

HEADER = Path(__file__).resolve().parents[1] / "include" / "clb200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(clb_[a-z0-9_]+)\s*\(", text)))


def test_library_builds_and_exports_every_declared_symbol():
    build.build_library()
    lib = ctypes.CDLL(str(build.LIBRARY))
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing


def test_python_signature_table_covers_the_header():
    assert sorted(backend.SIGNATURES) == declared_functions()


def test_load_library_sets_signatures_and_pure_helpers():
    lib = backend.load_library()
    assert lib.clb_abi_version() == 8
    for count in (0, 1, 4096, 4097, 16777216):
        assert lib.clb_scan_scratch_bytes(count) == backend.Backend.scan_scratch_bytes_static(count)
    assert lib.clb_mg_residual_partials(1000) == 4
    d = (ctypes.c_float * 3)()
    assert lib.clb_voxelise_direction(d) == 0
    assert abs(d[0] ** 2 + d[1] ** 2 + d[2] ** 2 - 1.0) < 1e-6


def test_hierarchy_struct_layout():
    # int32 levels (0), int32[16][3] (4..196), float delta (196), int32 fp16_level (200), then
    # 8-byte-aligned pointers: op0 at 208, the five pointer tables, int32 sweep[16], the three FP16
    # pointers, the tile table, the tile counts, the int32 zero_outside flag (padded to 8 bytes), the
    # two fused-tile pointers, the cluster lists, the float prolong_scale and the three int32 coarse
    # smoothing fields
    assert backend.MGHierarchy.delta.offset == 196
    assert backend.MGHierarchy.fp16_level.offset == 200
    assert backend.MGHierarchy.op0.offset == 208
    assert backend.MGHierarchy.p.offset == 216
    assert backend.MGHierarchy.fp16_scale.offset == 216 + 5 * 16 * 8 + 16 * 4
    tiles = 216 + 5 * 16 * 8 + 16 * 4 + 3 * 8
    assert backend.MGHierarchy.tiles.offset == tiles
    assert backend.MGHierarchy.zero_outside.offset == tiles + 16 * 8 + 8
    assert backend.MGHierarchy.fused_tiles.offset == tiles + 16 * 8 + 8 + 8
    assert backend.MGHierarchy.cluster_lists.offset == tiles + 16 * 8 + 8 + 8 + 2 * 8
    assert backend.MGHierarchy.prolong_scale.offset == tiles + 16 * 8 + 8 + 8 + 3 * 8
    assert backend.MGHierarchy.coarse_post_smooth.offset == tiles + 16 * 8 + 8 + 8 + 3 * 8 + 12
    assert ctypes.sizeof(backend.MGHierarchy) == tiles + 16 * 8 + 8 + 8 + 5 * 8


def test_tuned_preconditioner_settings_agree():
    """The benchmark's other cases run the library's tuned preconditioner settings."""
    import importlib.util

    from continuum_liquid_b200 import pressure_solve, solver

    spec = importlib.util.spec_from_file_location("bench_module", Path(__file__).resolve().parents[1] / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    assert bench.TUNED_WCYCLE == pressure_solve.TUNED_PRECONDITIONER
    solver.StepOptions(tol=1e-6, **pressure_solve.TUNED_PRECONDITIONER)  # every key is an option


def test_backend_without_gpu_fails_loudly(monkeypatch):
    import pytest
    import torch

    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    with pytest.raises(RuntimeError, match="CUDA"):
        backend.Backend(0)


def test_struct_layouts_match_the_c_compiler(tmp_path):
    """sizeof/offsetof of the header's structs, as gcc lays them out, against the ctypes mirrors."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or "/usr/bin/gcc"
    root = Path(__file__).resolve().parents[1]
    src = tmp_path / "layout.c"
    fields = {
        "clb_mg_hierarchy": ["fp16_level", "op0", "sweep", "fp16_scale", "rhs_norms", "fp16_inexact", "tiles",
                             "tile_counts", "zero_outside", "fused_tiles", "cluster_lists", "prolong_scale",
                             "coarse_smoothing", "coarse_post_smooth"],
        "clb_batch_scene": ["base", "particle_base", "delta", "upper", "pad"],
        "clb_batch_list": ["start", "count", "total"],
        "clb_batch": ["geom_host", "particles", "cells", "colour0", "sweep0", "bottom_smem", "op0", "op",
                      "prolong_scale", "coarse_smoothing", "coarse_post_smooth"],
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "clb200.h"', "int main(void) {"]
    for struct, names in fields.items():
        lines.append(f'printf("{struct} size %zu\\n", sizeof({struct}));')
        for n in names:
            lines.append(f'printf("{struct} {n} %zu\\n", offsetof({struct}, {n}));')
    lines.append("return 0; }")
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", str(root / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    mirrors = {"clb_mg_hierarchy": backend.MGHierarchy, "clb_batch_scene": backend.BatchScene,
               "clb_batch_list": backend.BatchList, "clb_batch": backend.Batch}
    for line in filter(None, out):
        struct, name, value = line.split()
        m = mirrors[struct]
        got = ctypes.sizeof(m) if name == "size" else getattr(m, name).offset
        assert got == int(value), (struct, name, got, value)
