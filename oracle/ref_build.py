"""Builds the reference's own OpenCL kernels for the host CPU into oracle/_ref/. Test infrastructure.

The reference (Continuum Liquid) runs its solver as OpenCL C programs, `Solver/Kernel/OpenCL/*.cl`,
compiled at run time by pyopencl (`Solver/Kernel/helper.py:22-48`). No OpenCL platform exists here,
and the OpenCL C does not compile as C++ as written. This recipe reads each program from the
reference checkout, applies a fixed list of mechanical rewrites, and compiles the result with g++
against `oracle/clshim.h` (the OpenCL C subset the programs use) and `oracle/clshim_runtime.cpp`:

1. `#include "X.cl"` is replaced by the (rewritten) text of X.cl from the same directory;
2. vector literals `(float3)(...)`, `(int3)(...)`, `(float4)(...)` become the calls
   `clshim_float3(...)`, `clshim_int3(...)`, `clshim_float4(...)`;
3. `#include "clshim.h"` is put first, the `-D` options the host passes to the program build are
   turned into `#define`s (those the program names), and one `CLSHIM_REGISTER(name, uses_barrier)` line is appended per
   `__kernel` (uses_barrier when its body calls `barrier(`).

Nothing else is touched: the kernels' statements, their order and their arithmetic are the
reference's. Output goes only to oracle/_ref/ (ignored by git): the rewritten sources, for reading,
and one shared library per program, named by a hash of its source and build options.
`oracle/pyopencl_shim/` loads these libraries when the reference's host code builds a program.

    python oracle/ref_build.py [REFERENCE_ROOT]     # prebuilds every program of the checkout
"""

from __future__ import annotations

import hashlib
import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

ORACLE_DIR = Path(__file__).resolve().parent
OUT_DIR = ORACLE_DIR / "_ref"
DEFAULT_REFERENCE = Path(os.environ.get("CLB_REFERENCE_ROOT", "/root/reference"))
KERNEL_SUBDIR = Path("Solver") / "Kernel" / "OpenCL"
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-w"]

_LITERAL = re.compile(r"\(\s*(float|int|uint|uchar)([2348]|16)\s*\)\s*\(")
_INCLUDE = re.compile(r'^\s*#\s*include\s+"([^"]+)"\s*$', re.MULTILINE)
_KERNEL = re.compile(r"__kernel\s+void\s+(\w+)\s*\(")


def _compiler() -> str:
    for candidate in ("/usr/bin/g++", shutil.which("g++")):
        if candidate and Path(candidate).exists():
            return candidate
    raise RuntimeError("g++ not found")


def _inline_includes(source: str, include_dirs: list[Path], seen: set[str]) -> str:
    def replace(match: re.Match) -> str:
        name = match.group(1)
        for directory in include_dirs:
            path = directory / name
            if path.exists():
                if str(path) in seen:
                    return ""
                seen.add(str(path))
                return _inline_includes(path.read_text(encoding="utf-8"), include_dirs, seen)
        raise FileNotFoundError(f"include {name!r} not found in {include_dirs}")

    return _INCLUDE.sub(replace, source)


def _kernel_bodies(source: str) -> dict[str, str]:
    """Kernel name -> its body text (brace-matched from the signature)."""
    bodies = {}
    for match in _KERNEL.finditer(source):
        start = source.index("{", match.end())
        depth, i = 0, start
        while True:
            if source[i] == "{":
                depth += 1
            elif source[i] == "}":
                depth -= 1
                if depth == 0:
                    break
            i += 1
        bodies[match.group(1)] = source[start : i + 1]
    return bodies


def parse_options(options) -> tuple[list[tuple[str, str]], list[Path]]:
    """The -D and -I options of a pyopencl Program.build call."""
    defines, include_dirs = [], []
    tokens = []
    for option in options or ():
        tokens.extend(re.findall(r'-[DI]\s*"[^"]*"|-[DI]\s*\S+|\S+', str(option)))
    for token in tokens:
        if token.startswith("-D"):
            body = token[2:].strip()
            name, _, value = body.partition("=")
            defines.append((name, value or "1"))
        elif token.startswith("-I"):
            include_dirs.append(Path(token[2:].strip().strip('"')))
    return defines, include_dirs


def translate(source: str, defines=(), include_dirs=()) -> tuple[str, dict[str, bool]]:
    """OpenCL C program text -> C++ text and {kernel name: uses a barrier}."""
    text = _inline_includes(source, list(include_dirs), set())
    text = _LITERAL.sub(lambda m: f"clshim_{m.group(1)}{m.group(2)}(", text)
    kernels = {name: "barrier(" in body for name, body in _kernel_bodies(text).items()}
    # a define the program never names changes nothing; leaving it out keeps the cache key stable
    used = [(n, v) for n, v in defines if re.search(rf"\b{re.escape(n)}\b", text)]
    head = ['#include "clshim.h"'] + [f"#define {name} {value}" for name, value in used]
    tail = [f"CLSHIM_REGISTER({name}, {int(uses)})" for name, uses in kernels.items()]
    return "\n".join(head) + "\n" + text + "\n" + "\n".join(tail) + "\n", kernels


def build_program(source: str, options=(), name: str = "program") -> Path:
    """Translates and compiles one program (cached by content); returns the shared library."""
    defines, include_dirs = parse_options(options)
    cpp, _ = translate(source, defines, include_dirs)
    runtime = (ORACLE_DIR / "clshim_runtime.cpp").read_text()
    header = (ORACLE_DIR / "clshim.h").read_text()
    digest = hashlib.sha256((cpp + runtime + header + " ".join(CXXFLAGS)).encode()).hexdigest()[:16]
    OUT_DIR.mkdir(exist_ok=True)
    existing = sorted(OUT_DIR.glob(f"lib*_{digest}.so"))
    if existing:
        return existing[0]
    library = OUT_DIR / f"lib{name}_{digest}.so"
    cpp_path = OUT_DIR / f"{name}_{digest}.cpp"
    cpp_path.write_text(cpp)
    command = [_compiler(), *CXXFLAGS, f"-I{ORACLE_DIR}", "-o", str(library) + ".tmp", str(cpp_path),
               str(ORACLE_DIR / "clshim_runtime.cpp")]
    result = subprocess.run(command, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"g++ failed on {name}:\n{result.stderr[-4000:]}")
    os.replace(str(library) + ".tmp", library)
    return library


def build_reference(reference_root: Path = DEFAULT_REFERENCE) -> list[Path]:
    """Prebuilds every program of the reference checkout (the host's -D options name nothing the
    programs use, so the libraries are the ones its Program.build calls load)."""
    kernel_dir = reference_root / KERNEL_SUBDIR
    if not kernel_dir.is_dir():
        raise FileNotFoundError(f"no reference kernels at {kernel_dir}")
    options = [f'-I "{kernel_dir}"']
    built = []
    for path in sorted(kernel_dir.glob("*.cl")):
        if path.name == "helper.cl":
            continue
        built.append(build_program(path.read_text(encoding="utf-8"), options, path.stem))
    return built


if __name__ == "__main__":
    root = Path(sys.argv[1]) if len(sys.argv) > 1 else DEFAULT_REFERENCE
    for library in build_reference(root):
        print(library)
