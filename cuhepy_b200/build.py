"""Build the sm_100a shared libraries in-tree (``python -m cuhepy_b200.build``).

Each library is one nvcc invocation with ``-gencode arch=compute_100a,code=sm_100a``;
outputs go to ``cuhepy_b200/lib/`` so they travel with the source tree.
A library is rebuilt only when one of its sources is newer than the output.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
INCLUDE = PKG.parent / "include"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-shared", "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
]

LIBRARIES = {
    "libcuhe_b200.so": {
        "sources": ["cuhe_paillier.cu"],
        "depends": ["bigint_group.cuh", "paillier_kernels.cuh", "host_bigint.h"],
        "headers": ["cuhe_paillier.h"],
    },
    "libcuhe_bfv_b200.so": {
        "sources": ["cuhe_bfv.cu"],
        "depends": ["bfv_arith.cuh", "bfv_host.h", "bfv_kernels.cuh"],
        "headers": ["cuhe_bfv.h", "cuhe_paillier.h"],
    },
}


def nvcc() -> str:
    for candidate in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if candidate and Path(candidate).exists():
            return candidate
    raise RuntimeError("nvcc not found")


def _stale(output: Path, inputs: list[Path]) -> bool:
    if not output.exists():
        return True
    mtime = output.stat().st_mtime
    return any(p.stat().st_mtime > mtime for p in inputs)


def build_library(name: str, force: bool = False, verbose: bool = False) -> Path:
    spec = LIBRARIES[name]
    LIB.mkdir(exist_ok=True)
    out = LIB / name
    inputs = [CSRC / s for s in spec["sources"] + spec["depends"]] + [INCLUDE / h for h in spec["headers"]]
    if not force and not _stale(out, inputs):
        return out
    tmp = out.with_suffix(".so.tmp")
    cmd = [nvcc(), *NVCC_FLAGS, "-I", str(INCLUDE), "-o", str(tmp), *[str(CSRC / s) for s in spec["sources"]]]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    tmp.replace(out)
    return out


def build_all(force: bool = False, verbose: bool = False) -> list[Path]:
    return [build_library(name, force, verbose) for name in LIBRARIES]


if __name__ == "__main__":
    force = "--force" in sys.argv
    for path in build_all(force=force, verbose="-v" in sys.argv):
        print(path)
