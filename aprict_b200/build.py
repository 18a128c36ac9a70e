"""Build libaprict_b200.so (all CUDA sources under csrc/) for sm_100a, in-tree.

Usage: ``python -m aprict_b200.build`` (or ``build()`` from Python). The shared
library is written next to this file so that it travels with the package; a
rebuild happens only when a source or header is newer than the library.
"""

from __future__ import annotations

import concurrent.futures
import os
import pathlib
import shutil
import subprocess
import sys

PKG_DIR = pathlib.Path(__file__).resolve().parent
REPO_DIR = PKG_DIR.parent
CSRC = PKG_DIR / "csrc"
INCLUDE = REPO_DIR / "include"
LIB_PATH = PKG_DIR / "libaprict_b200.so"
BUILD_DIR = PKG_DIR / "_build"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-Xptxas",
    "-warn-spills",
]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not pathlib.Path(cand).exists():
        msg = "nvcc not found; install the CUDA toolkit to build aprict_b200"
        raise RuntimeError(msg)
    return cand


def sources() -> list[pathlib.Path]:
    return sorted(CSRC.glob("*.cu"))


def _inputs() -> list[pathlib.Path]:
    return sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def needs_rebuild() -> bool:
    if not LIB_PATH.exists():
        return True
    t = LIB_PATH.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _inputs())


def build(*, force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> pathlib.Path:
    """Compile every ``csrc/*.cu`` to an object and link ``libaprict_b200.so``."""
    if not force and not needs_rebuild():
        return LIB_PATH
    nvcc = _nvcc()
    BUILD_DIR.mkdir(exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []

    def compile_one(src: pathlib.Path) -> str:
        obj = BUILD_DIR / (src.stem + ".o")
        cmd = [nvcc, *ARCH_FLAGS, *NVCC_FLAGS, *extra, f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        res = subprocess.run(cmd, capture_output=True, text=True, check=False)
        if res.returncode != 0 or verbose or ptxas_verbose:
            sys.stderr.write(f"== {src.name}\n" + res.stdout + res.stderr)
        if res.returncode != 0:
            msg = f"nvcc failed on {src.name}"
            raise RuntimeError(msg)
        return str(obj)

    # one nvcc per source file, in parallel
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(sources()), os.cpu_count() or 1))) as ex:
        objs = list(ex.map(compile_one, sources()))
    tmp = LIB_PATH.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH_FLAGS, "-shared", "-o", str(tmp), *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    res = subprocess.run(cmd, capture_output=True, text=True, check=False)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        msg = "linking libaprict_b200.so failed"
        raise RuntimeError(msg)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv, ptxas_verbose="--ptxas" in sys.argv)
    print(LIB_PATH)
