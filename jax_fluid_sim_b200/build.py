"""Build the in-tree CUDA library ``libdgb200.so`` for sm_100a with nvcc.

    python -m jax_fluid_sim_b200.build [--verbose]

The library is a plain C-ABI shared object (see ``include/dgb200.h``) loaded by
ctypes; it is built in the package directory so that it travels with the tree.
"""

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
LIB = PKG / "libdgb200.so"
SOURCES = [PKG / "csrc" / "capi.cu", PKG / "csrc" / "noalloc.cu", PKG / "csrc" / "chemistry.cu",
           PKG / "csrc" / "raster.cu", PKG / "csrc" / "setup.cpp"]
DEPENDS = sorted((PKG / "csrc").glob("*.c*")) + [ROOT / "include" / "dgb200.h"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (Path(cand).exists() or cand == "nvcc"):
            return cand
    raise RuntimeError("nvcc not found")


def up_to_date():
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in DEPENDS)


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    cmd = [nvcc(), "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
           "-shared", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include"), "-o", str(LIB)]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [str(s) for s in SOURCES]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + proc.stdout + proc.stderr)
    if verbose:
        sys.stderr.write(proc.stderr)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose="--verbose" in sys.argv)
    print(LIB)
