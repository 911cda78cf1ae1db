"""The ctypes binding documented in INTEGRATION.md, executed as written.

CPU: its struct definitions match the sizes the built library reports
(ug_struct_sizes), so ug_pack_create never reads past a caller's struct.
GPU: its run_job gives the same (N, attempts) as the braid_cuda command line
that braidlab.engine builds for the same Job.
"""

import os
import re
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "universe-generator_b200", "bin")


def _stub() -> dict:
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    block = re.search(r"```python\n(import ctypes as C\n.*?)```", text, re.S).group(1)
    ns: dict = {}
    cwd = os.getcwd()
    os.chdir(ROOT)  # the stub loads the library by its repository-relative path
    try:
        exec(compile(block, "INTEGRATION.md", "exec"), ns)
    finally:
        os.chdir(cwd)
    return ns


def test_stub_structs_match_the_library(ug):
    import ctypes as C

    from ugb200 import _lib

    ns = _stub()  # asserts the three sizes itself
    sizes = (C.c_int64 * 7)()
    assert _lib.load().ug_struct_sizes(sizes, 7) == 7
    assert C.sizeof(ns["Cfg"]) == sizes[0] == C.sizeof(_lib.UniverseCfg)
    assert C.sizeof(ns["Opts"]) == sizes[1] == C.sizeof(_lib.RunOpts)
    assert C.sizeof(ns["Stats"]) == sizes[2] == C.sizeof(_lib.Stats)
    assert sizes[3] == C.sizeof(_lib.KernelTimes)
    assert sizes[4] == 20  # the BRF1 hit record


@pytest.mark.gpu
@pytest.mark.parametrize("terms", [2, 3, 16])
def test_stub_run_job_equals_braid_cuda(ug, terms):
    from braidlab.config import Job
    from braidlab.engine import binary_name, build_command, parse_done

    job = Job(dim=2, t=16, seed=5, accept_rate=1e-9, max_attempts=30000.0, terms=terms)
    ns = _stub()
    n, att = ns["run_job"](job)
    cmd = build_command(job, binary_name(job.dim, job.terms), os.devnull)
    r = subprocess.run([sys.executable, os.path.join(BIN, cmd[0]), *cmd[1:]], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert (n, att) == parse_done(r.stderr)
