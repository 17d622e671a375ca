"""Build liboal.so (the sm_100a CUDA library) in-tree with nvcc.

``python -m openaerolab_alpha_01_b200.build`` compiles every ``csrc/*.cu`` and ``csrc/*.cpp`` into
``openaerolab_alpha_01_b200/liboal.so``. The library links the CUDA runtime statically, so the
built file is self-contained and travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "liboal.so"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: the scalar arithmetic of the kernels fuses only the multiply-adds written explicitly
# (the bit-exact D3Q39, octree and SVV paths rely on it); packed f32x2 code agrees to rounding.
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "--expt-relaxed-constexpr", "-fmad=false", "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found")
    return path


def sources() -> list[Path]:
    """CUDA sources and the host-only C++ sources (the mesh generator), all compiled by nvcc."""
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None,
          out: Path | None = None, objdir: Path | None = None) -> Path:
    """Compile the CUDA sources into liboal.so (objects under csrc/_build/), or into `out` with
    extra nvcc flags (tuning variants)."""
    srcs = sources()
    headers = list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    lib = Path(out) if out else LIB
    objdir = Path(objdir) if objdir else CSRC / "_build"
    objdir.mkdir(parents=True, exist_ok=True)
    objs = []
    procs = []
    for s in srcs:
        o = objdir / (s.name.replace(".", "_") + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc(), *ARCH_FLAGS, *NVCC_FLAGS, *(extra or []), "-I", str(INCLUDE), "-c", str(s), "-o", str(o)]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for s, p in procs:
        out, _ = p.communicate()
        if verbose and out:
            sys.stdout.write(out)
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {s.name}:\n{out}")
    if force or _stale(lib, objs):
        cmd = [nvcc(), *ARCH_FLAGS, "-shared", "-o", str(lib), *map(str, objs)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}{r.stderr}")
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
