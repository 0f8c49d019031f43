"""Builds the sm_100a shared library liblpg_b200.so in-tree with nvcc.

Run as ``python -m litepgo_b200.build`` (or through ``__graft_entry__.build()``). The
library is written to litepgo_b200/_lib/ so that it travels with the source tree.
"""

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "csrc"
OUT_DIR = HERE / "_lib"
LIB = OUT_DIR / "liblpg_b200.so"
INCLUDE = HERE.parent / "include"

SOURCES = ["lpg_plan.cpp", "lpg_veg.cpp", "lpg_assemble.cu", "lpg_solve.cu", "lpg_api.cu", "lpg_noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "--expt-relaxed-constexpr"]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build litepgo_b200")
    return path


def _stale():
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [SRC / s for s in SOURCES] + list(SRC.glob("*.h")) + list(SRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    deps.append(Path(__file__))
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(force=False, verbose=False, ptxas_info=False):
    """Compiles every CUDA/C++ source for sm_100a and links liblpg_b200.so; returns its path."""
    if not force and not _stale():
        return LIB
    OUT_DIR.mkdir(exist_ok=True)
    obj_dir = OUT_DIR / "obj"
    obj_dir.mkdir(exist_ok=True)
    cc = nvcc()
    extra = ["-Xptxas", "-v"] if ptxas_info else []

    def compile_one(name):
        src = SRC / name
        obj = obj_dir / (name + ".o")
        cmd = [cc, *ARCH, *FLAGS, *extra, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {name}:\n{r.stderr}")
        return obj, r.stderr

    with concurrent.futures.ThreadPoolExecutor(max_workers=min(4, os.cpu_count() or 1)) as pool:
        results = list(pool.map(compile_one, SOURCES))
    if verbose or ptxas_info:
        for (_, log), name in zip(results, SOURCES):
            if log.strip():
                print(f"--- {name}\n{log}", file=sys.stderr)
    objs = [str(o) for o, _ in results]
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [cc, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build(force=force, verbose=True, ptxas_info="--ptxas" in sys.argv))
