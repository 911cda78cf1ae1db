"""The index-guarded build (libug_checked.so: every data-dependent device index
checked against its buffer, the first violation recorded and reported as an
error) runs parity cases that reach the hash grid, group rounds, the coarsened
occupancy bitmaps and the tensor-core prefilter, and reports no violation.
This build stands in for compute-sanitizer, which is closed on this pool."""

import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, sys
sys.path[:0] = [ROOT, ROOT + "/universe-generator_b200"]
import numpy as np
import oracle as O
import ugb200
from ugb200 import _lib
assert _lib.LIB_PATH.endswith("libug_checked.so"), _lib.LIB_PATH
cases = [
    dict(dim=2, T=32, zgrid=1, excl=1, seed=11, attempts=60000, round_size=4096),
    dict(dim=3, T=200, zgrid=1, excl=1, seed=12, attempts=8000, round_size=2048),
    dict(dim=2, T=40, zgrid=1, excl=1, seed=13, attempts=40000, group_mode=2, round_size=4096),
]
out = []
for kw in cases:
    for prec, hashed in ((0, True), (1, False), (1, True)):
        u = ugb200.Universe(**kw)
        with ugb200.Packer([u], precision=prec, force_hash=hashed) as p:
            p.run()
            idx, gid = p.accepted(0)
        m = O.Model(dim=u.dim, T=u.T, zgrid=u.zgrid, excl=u.excl, seed=u.seed)
        r = O.pack(m, u.attempts, group_mode=u.group_mode)
        assert np.array_equal(idx, r.acc_idx) and np.array_equal(gid, r.gid), (kw, prec, hashed)
        out.append(len(idx))
print(json.dumps(out))
""".replace("ROOT", repr(ROOT))


def test_checked_build_reports_no_violation():
    lib = os.path.join(ROOT, "universe-generator_b200", "ugb200", "libug_checked.so")
    assert os.path.exists(lib), "libug_checked.so is not built (ugb200/build.py --checked)"
    env = {**os.environ, "UG_LIB": "checked"}
    r = subprocess.run([sys.executable, "-c", SCRIPT], capture_output=True, text=True, env=env, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    assert len(json.loads(r.stdout.strip().splitlines()[-1])) == 9
