"""Build recipe for libspexgpu.so (sm_100a) — compiled in-tree with nvcc.

The shared library is the product: every kernel and the C ABI declared in
include/spexgpu.h. It is linked against the static CUDA runtime so that it
loads next to any PyTorch build and on hosts without a GPU (where every call
returns SPX_ENODEV).
"""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libspexgpu.so"
INCLUDE = ROOT / "include"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "-Xptxas", "-warn-spills",
    "--expt-relaxed-constexpr",
    "-cudart", "static",
]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def needs_rebuild() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*")) + list(INCLUDE.glob("*.h")) + [Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps if p.is_file())


def build_library(force: bool = False, verbose: bool = False) -> Path:
    """Compile every .cu under csrc/ into libspexgpu.so (one nvcc call per file, then link)."""
    if not force and not needs_rebuild():
        return LIB
    nvcc = nvcc_path()
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    host_cc = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else None
    objs = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        cmd = [nvcc, *NVCC_FLAGS, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
        if host_cc:
            cmd[1:1] = ["-ccbin", host_cc]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    cmd = [nvcc, "-shared", "-cudart", "static", "-gencode", "arch=compute_100a,code=sm_100a",
           *objs, "-ldl", "-o", str(LIB) + ".tmp"]
    if host_cc:
        cmd[1:1] = ["-ccbin", host_cc]
    subprocess.run(cmd, check=True)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build_library(force=True, verbose=True)
    print(LIB)
