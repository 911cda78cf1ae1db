"""Engine command construction and result parsing (reference braidlab/engine.py:25-112).

The binaries are the B200 packer's drop-in executables in
``universe-generator_b200/bin`` (``braid_cuda``, ``braid_cuda3d`` and their ``_w150``
names), which accept the engines' flags and print the same ``done:`` line.
"""

from __future__ import annotations

import os
import re

from .config import Job

_DONE = re.compile(r"done:\s*N=(\d+)\s+in\s+(\d+)\s+attempts")

DEFAULT_MAX_WIGGLE = 9      # wiggle-term cap of the reference's default binaries
WIDE_MAX_WIGGLE = 149       # cap of the reference's wide binaries
WIDE_SUFFIX = "_w150"
BIN_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bin")


def binary_name(dim: int, terms: int = 2) -> str:
    """Executable for a spatial dimension; terms above the default cap take the
    wide name (the B200 packer has no compiled cap, both names run it)."""
    name = "braid_cuda" if dim == 2 else "braid_cuda3d"
    return name + WIDE_SUFFIX if terms - 1 > DEFAULT_MAX_WIGGLE else name


def binary_path(binary: str) -> str:
    """Absolute path of a drop-in executable."""
    return os.path.join(BIN_DIR, binary)


def binary_source(binary: str) -> str:
    """Source of a binary: the drop-in executables are scripts, nothing to compile."""
    return binary_path(binary)


def binary_build_flags(binary: str) -> str:
    return ""


def build_command(job: Job, binary: str, curve_path: str) -> list[str]:
    """argv of one packing run, flag for flag the reference's."""
    cmd = [binary, "-t", str(job.t), "--attempts", repr(job.max_attempts),
           "--uniform", "--torus", "--phase",
           "--seed", str(job.seed), "--until-accept-rate", repr(job.accept_rate)]
    if job.euclid:
        cmd.append("--euclid-collision")
    if job.sparse:
        cmd.append("--sparse")
    if job.terms != 2:
        cmd += ["--terms", str(job.terms)]
    if job.subpaths:
        cmd += ["--subpaths", "--sub-until-accept-rate", repr(job.accept_rate)]
        if job.sub_attempts:
            cmd += ["--sub-attempts", repr(job.sub_attempts)]
    cmd += ["--maxfreq", str(job.maxfreq), "--curve", curve_path]
    return cmd


def parse_done(text: str) -> tuple[int, int] | None:
    """(n_final, attempts) from ``done: N=<n> in <attempts> attempts``, or None."""
    m = _DONE.search(text)
    return (int(m.group(1)), int(m.group(2))) if m else None
