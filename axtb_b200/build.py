"""Build ``libaxtb_gpu.so`` in-tree for sm_100a (``python -m axtb_b200.build``)."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "csrc" / "axtb_gpu.cu"
OUT = HERE / "libaxtb_gpu.so"
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
         "-shared"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return [SRC] + sorted((HERE / "csrc").glob("*.cuh")) + [HERE / "csrc" / "params" / "gfn2_tables.h"] + \
        sorted((HERE.parent / "include").glob("*.h"))


def build(force: bool = False) -> Path:
    if not force and OUT.exists() and OUT.stat().st_mtime >= max(p.stat().st_mtime for p in sources()):
        return OUT
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [nvcc(), *FLAGS, "-o", str(tmp), str(SRC)]
    subprocess.run(cmd, check=True)
    tmp.replace(OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
