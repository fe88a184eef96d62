"""Build liblesgpu.so (sm_100a) in-tree with nvcc.

Each translation unit compiles in its own nvcc process; the objects are
linked into ``new_repo_b200/liblesgpu.so`` next to this file.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE.parent / "_build"
LIB = HERE / "liblesgpu.so"
SOURCES = ["spectral_inst.cu", "spectral_xfwd.cu", "spectral_xinv.cu", "spectral_ypass.cu", "solver.cu", "capi.cu", "mlp.cu", "noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fno-strict-aliasing",
         "--expt-relaxed-constexpr", "-I", str(HERE.parent / "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + list(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "lesgpu.h"]
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = [CSRC / s for s in SOURCES if (CSRC / s).exists()]
    objs = [BUILD / (s.stem + ".o") for s in srcs]
    cc = nvcc()

    def compile_one(pair):
        src, obj = pair
        if not _stale(obj, src) and not ptxas_info:
            return ""
        cmd = [cc, *ARCH, *FLAGS, "-c", str(src), "-o", str(obj)]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stderr}")
        return r.stderr

    with ThreadPoolExecutor(max_workers=len(srcs)) as ex:
        logs = list(ex.map(compile_one, zip(srcs, objs)))
    if verbose:
        for l in logs:
            if l:
                print(l)
    if not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        # link to a temporary name and rename: a process loading the library
        # meanwhile sees the old file or the new one, never a partial one
        tmp = LIB.with_name(LIB.name + ".tmp")
        cmd = [cc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="-v" in sys.argv))
