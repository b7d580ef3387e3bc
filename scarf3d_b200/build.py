"""Build libscarf3d_b200.so in-tree (sm_100a device code, C++17 host code).

Device code: nvcc -gencode arch=compute_100a,code=sm_100a.
Host code: g++ with -ffp-contract=off so every single-precision operation of
the sampler and setup rounds as the reference's Fortran statements do.
The CUDA runtime is linked statically so the library only needs the driver.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libscarf3d_b200.so"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
CXX = os.environ.get("CXX", shutil.which("g++") or "g++")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = [f"-I{ROOT / 'include'}", f"-I{CSRC}"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                     "-Xcompiler", "-ffp-contract=off", "-Xptxas", "-warn-spills"] + INCLUDES
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-Wall",
             f"-I{CUDA_HOME / 'include'}"] + INCLUDES


def _needs(obj: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose_ptxas: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted((ROOT / "include").glob("*.h"))
    objs = []
    for src in sorted(CSRC.glob("*.cu")):
        obj = BUILD / (src.stem + ".o")
        if _needs(obj, [src] + headers) or verbose_ptxas:
            flags = NVCC_FLAGS + (["-Xptxas", "-v"] if verbose_ptxas else [])
            _run([NVCC] + flags + ["-c", str(src), "-o", str(obj)])
        objs.append(obj)
    for src in sorted(CSRC.glob("*.cpp")):
        obj = BUILD / (src.stem + ".o")
        if _needs(obj, [src] + headers):
            _run([CXX] + CXX_FLAGS + ["-c", str(src), "-o", str(obj)])
        objs.append(obj)
    if _needs(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", str(LIB)] + [str(o) for o in objs]
             + ["-lpthread"])
    build_standalone()
    build_fbind()
    return LIB


FBIND_SRC = PKG / "fbind" / "scarf3d_fbind.cpp"
FBIND = PKG / "libscarf3d_b200_fbind.so"


def build_fbind() -> Path:
    """The reference's Fortran BIND(C) routine names (struct_initialize,
    execute, ...) as a separate shim over the library."""
    if _needs(FBIND, [FBIND_SRC, LIB] + sorted((ROOT / "include").glob("*.h"))):
        _run([CXX, "-O2", "-std=c++17", "-Wall", "-shared", "-fPIC"] + INCLUDES + [str(FBIND_SRC), f"-L{PKG}",
              "-lscarf3d_b200", "-Wl,-rpath,$ORIGIN", "-o", str(FBIND)])
    return FBIND


STANDALONE_SRC = PKG / "standalone" / "scarf3d_standalone.cpp"
STANDALONE = PKG / "scarf3d_standalone"


def build_standalone() -> Path:
    """The keyword-file driver (counterpart of the reference's standalone
    application), linked against the library next to it."""
    if _needs(STANDALONE, [STANDALONE_SRC, LIB] + sorted((ROOT / "include").glob("*.h"))):
        _run([CXX, "-O2", "-std=c++17", "-Wall"] + INCLUDES + [str(STANDALONE_SRC), f"-L{PKG}", "-lscarf3d_b200",
              "-Wl,-rpath,$ORIGIN", "-o", str(STANDALONE)])
    return STANDALONE


def build_oracle() -> Path:
    """Build the CPU oracle used by the tests (test infrastructure)."""
    _run(["make", "-C", str(ROOT / "oracle"), "-s"])
    return ROOT / "oracle" / "liboracle_srm.so"


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv)
    build_oracle()
