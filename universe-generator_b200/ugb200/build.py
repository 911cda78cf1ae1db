"""Compile the packer's CUDA sources into the in-tree shared library libug.so.

nvcc cross-compiles for sm_100a (no GPU needed).  The library is built next
to this file so it travels with the source tree.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "csrc")
LIB = os.path.join(HERE, "libug.so")
SOURCES = ["ug_host.cu", "ug_kernels.cu", "ug_mixed.cu", "ug_frames.cu", "ug_noalloc.cu"]
FLAGS = [
    "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr",
]


def sources() -> list[str]:
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(os.path.dirname(os.path.dirname(HERE)), "include", "ug.h"))
    return all(os.path.getmtime(p) <= t for p in deps if os.path.exists(p))


LIB_CHECKED = os.path.join(HERE, "libug_checked.so")


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> str:
    """Build libug.so, or with checked=True the index-guarded libug_checked.so
    (separate device compilation so the guard record has one definition)."""
    lib = LIB_CHECKED if checked else LIB
    if not force and not checked and up_to_date():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    extra = ["-DUG_CHECKED", "-rdc=true"] if checked else []
    cmd = [nvcc, *FLAGS, *extra, "-o", lib + ".tmp", *sources()]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True, cwd=CSRC)
    os.replace(lib + ".tmp", lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv, checked="--checked" in sys.argv))
