"""Build the in-tree CUDA library ``libdgb200.so`` for sm_100a with nvcc.

    python -m jax_fluid_sim_b200.build [--verbose]

The library is a plain C-ABI shared object (see ``include/dgb200.h``) loaded by
ctypes; it is built in the package directory so that it travels with the tree.
Each translation unit is compiled to its own object in parallel (``_build/``), and
only the units whose sources changed are recompiled; then nvcc links the library.
"""

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
LIB = PKG / "libdgb200.so"
OBJ = PKG / "_build"
SOURCES = [PKG / "csrc" / "capi.cu", PKG / "csrc" / "tc_volume.cu",
           PKG / "csrc" / "noalloc.cu", PKG / "csrc" / "chemistry.cu", PKG / "csrc" / "raster.cu",
           PKG / "csrc" / "setup.cpp", PKG / "csrc" / "mesh_io.cpp"]
HEADERS = sorted((PKG / "csrc").glob("*.cuh")) + sorted((PKG / "csrc").glob("*.h")) + [ROOT / "include" / "dgb200.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (Path(cand).exists() or cand == "nvcc"):
            return cand
    raise RuntimeError("nvcc not found")


def _object(src):
    return OBJ / (src.name + ".o")


def _stale(src, newest_header):
    obj = _object(src)
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or newest_header > t


def up_to_date():
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in SOURCES + HEADERS)


def _compile(src, verbose):
    cmd = [nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include"),
           "-c", str(src), "-o", str(_object(src))]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n" + proc.stdout + proc.stderr)
    return proc.stderr


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    OBJ.mkdir(exist_ok=True)
    newest_header = max(p.stat().st_mtime for p in HEADERS)
    todo = [s for s in SOURCES if force or _stale(s, newest_header)]
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as pool:
        logs = list(pool.map(lambda s: _compile(s, verbose), todo))
    if verbose:
        for text in logs:
            sys.stderr.write(text)
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB)] + [str(_object(s)) for s in SOURCES]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + proc.stdout + proc.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv or "--verbose" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
