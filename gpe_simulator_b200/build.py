"""Build ``libgpe_ssf.so`` in-tree with nvcc for sm_100a.

The library is the product: the Python package loads it through ctypes and
fails loudly when it is missing.  Sources are compiled in parallel (one
translation unit per precision plus the host/C-ABI unit) and linked with the
static CUDA runtime.
"""

import concurrent.futures
import os
from pathlib import Path
import shutil
import subprocess

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libgpe_ssf.so"
OBJ = PKG / "_build"

FAST_SIZES = (32, 48, 64, 96, 128, 160, 256)
SOURCES = (["gpe_ssf.cu", "gpe_sweep_f32.cu", "gpe_sweep_f64.cu", "gpe_noalloc.cu", "gpe_fast_dispatch.cu"]
           + [f"gpe_fast_{p}_{n}.cu" for p in ("f32", "f64") for n in FAST_SIZES] + ["gpe_fast_f32_512.cu"])
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(INCLUDE),
         "--expt-relaxed-constexpr"]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libgpe_ssf.so")
    return exe


def _inputs():
    files = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h"))
    files += list(INCLUDE.glob("*.h")) + [Path(__file__)]
    return files


def up_to_date():
    if not LIB.exists():
        return False
    stamp = LIB.stat().st_mtime
    return all(f.stat().st_mtime <= stamp for f in _inputs())


def build(force=False, verbose=False):
    """Compile every CUDA source for sm_100a and link ``libgpe_ssf.so``."""
    if not force and up_to_date():
        return LIB
    exe = nvcc()
    OBJ.mkdir(exist_ok=True)

    def compile_one(src):
        obj = OBJ / (Path(src).stem + ".o")
        cmd = [exe, *ARCH, *FLAGS, "-c", str(CSRC / src), "-o", str(obj)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
        if verbose:
            print(res.stdout, res.stderr)
        return obj

    workers = min(len(SOURCES), os.cpu_count() or 1)
    with concurrent.futures.ThreadPoolExecutor(workers) as pool:
        objs = list(pool.map(compile_one, SOURCES))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [exe, *ARCH, "-shared", "-o", str(tmp), *map(str, objs)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=False))
