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


def _objects_dir() -> str:
    d = os.path.join(HERE, "_build")
    os.makedirs(d, exist_ok=True)
    return d


def _compile_one(src: str, verbose: bool) -> str:
    """Compiles one translation unit to an object under sdddst_b200/_build/
    when the object is older than the source or any header."""
    obj = os.path.join(_objects_dir(), os.path.basename(src) + ".o")
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    headers += glob.glob(os.path.join(HOST, "include", "*.h")) + glob.glob(os.path.join(HOST, "include", "*", "*.h"))
    headers.append(os.path.join(ROOT, "include", "sdddst_b200.h"))
    if os.path.exists(obj) and all(os.path.getmtime(d) <= os.path.getmtime(obj) for d in [src] + headers):
        return obj
    flags = [f for f in FLAGS if f != "-shared"]
    cmd = [nvcc()] + ARCH + flags + ["-I", os.path.join(ROOT, "include"), "-I", os.path.join(HOST, "include"),
                                     "-c", src, "-o", obj + ".tmp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=HERE)
    os.replace(obj + ".tmp", obj)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the library if any source is newer than it; returns its path.
    Translation units compile in parallel to objects, then one link."""
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    srcs = sources()
    if force:
        for s in srcs:
            o = os.path.join(_objects_dir(), os.path.basename(s) + ".o")
            if os.path.exists(o):
                os.remove(o)
    with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
        objs = list(ex.map(lambda s: _compile_one(s, verbose), srcs))
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", tmp] + objs + ["-lz"]
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


CLI_SRC = os.path.join(HERE, "cli", "sdddst_main.cpp")
CLI = os.path.join(HERE, "sdddst")


def build_cli(force: bool = False, verbose: bool = False) -> str:
    """Compile the `sdddst` command-line drop-in against the engine library."""
    lib = build(verbose=verbose)
    if not force and os.path.exists(CLI) and os.path.getmtime(CLI) >= max(os.path.getmtime(lib),
                                                                         os.path.getmtime(CLI_SRC)):
        return CLI
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    cmd = [cxx, "-O2", "-std=c++17", "-I", os.path.join(HOST, "include"), "-I", os.path.join(ROOT, "include"),
           CLI_SRC, "-o", CLI + ".tmp", "-L", HERE, "-lsdddst_b200", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=HERE)
    os.replace(CLI + ".tmp", CLI)
    return CLI


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    build_python_module(force="--force" in sys.argv, verbose=True)
    build_cli(force="--force" in sys.argv, verbose=True)
