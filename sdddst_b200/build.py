"""Builds the engine's shared library in-tree: ``sdddst_b200/libsdddst_b200.so``
from ``sdddst_b200/csrc/*.cu`` for sm_100a only, with nvcc.

    python -m sdddst_b200.build [--force]
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsdddst_b200.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-shared"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


HOST = os.path.join(HERE, "host")
PYMOD_SRC = os.path.join(HERE, "python", "pysdddstcore.cpp")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu"))) + sorted(glob.glob(os.path.join(HOST, "src", "*.cpp")))


def pymod_path() -> str:
    import sysconfig
    return os.path.join(HERE, "PySdddstCore" + (sysconfig.get_config_var("EXT_SUFFIX") or ".so"))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    deps += glob.glob(os.path.join(HOST, "include", "*.h")) + glob.glob(os.path.join(HOST, "include", "*", "*.h"))
    deps.append(os.path.join(ROOT, "include", "sdddst_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the library if any source is newer than it; returns its path."""
    if not force and not _stale():
        return LIB
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + FLAGS + ["-I", os.path.join(ROOT, "include"), "-I", os.path.join(HOST, "include"),
                                     "-o", tmp] + sources()
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=HERE)
    os.replace(tmp, LIB)
    return LIB


def build_python_module(force: bool = False, verbose: bool = False) -> str:
    """Compile the PySdddstCore module (pybind11) against the engine library."""
    import sysconfig
    import pybind11
    lib = build(verbose=verbose)
    out = pymod_path()
    if not force and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(lib),
                                                                          os.path.getmtime(PYMOD_SRC)):
        return out
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    cmd = [cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-I", pybind11.get_include(),
           "-I", sysconfig.get_paths()["include"], "-I", os.path.join(HOST, "include"),
           "-I", os.path.join(ROOT, "include"), PYMOD_SRC, "-o", out + ".tmp", "-L", HERE, "-lsdddst_b200",
           "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=HERE)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    build_python_module(force="--force" in sys.argv, verbose=True)
