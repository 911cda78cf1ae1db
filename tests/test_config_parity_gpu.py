"""GPU parity at the measured workloads' full sizes: the packer's accepted sets
against the oracle's, for c0, c1, c2, c4, all 256 universes of c3 (each to its
attempt cap), the reference conventions, the reference's xoshiro stream and the
windowed stops.

The oracle's results are committed fixtures (tests/golden/config_parity.json,
made by tests/golden/make_config_golden.py on the CPU): per case the accepted
count, the attempts and the SHA-256 of the accepted candidate indices (int64,
admission order) and group labels (int32).  Both precision modes must
reproduce them bit for bit.  These cases reach the code paths that only large
runs use: hash-grid growth, coarsened occupancy bitmaps of 3+1 universes at
large T, conflict-list overflow and survivor-capacity truncation of crowded
rounds.
"""

import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "config_parity.json")) as _f:
    CASES = json.load(_f)["cases"]

SINGLE = sorted(k for k in CASES if not k.startswith("c3/"))


def _sha(a, dt) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dt).tobytes()).hexdigest()


def _check(name, st, idx, gid):
    ref = CASES[name]
    got = (len(idx), st.n_unique, st.n_sub, st.attempts, st.phase1_end)
    want = (ref["n"], ref["n_unique"], ref["n_sub"], ref["attempts"], ref["phase1_end"])
    assert got == want, f"{name}: (n, n_unique, n_sub, attempts, phase1_end) {got} != {want}"
    assert _sha(idx, "<i8") == ref["idx_sha256"], \
        f"{name}: accepted indices differ (head {list(idx[:4])} vs {ref['head']}, tail {list(idx[-4:])} vs {ref['tail']})"
    assert _sha(gid, "<i4") == ref["gid_sha256"], f"{name}: group labels differ"


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name", SINGLE)
def test_workload_case(ug, name, precision):
    u = ug.Universe(**CASES[name]["universe"])
    with ug.Packer([u], precision=precision) as p:
        p.run()
        st = p.stats(0)
        assert st.done
        idx, gid = p.accepted(0)
    _check(name, st, idx, gid)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_c3_all_universes_batched(ug, precision):
    """All 256 universes of c3 in one batch (the measured configuration), each run to
    its attempt cap, against the oracle's per-universe fixtures."""
    names = sorted((k for k in CASES if k.startswith("c3/")), key=lambda k: int(k.split("/")[1]))
    assert len(names) == 256
    us = [ug.Universe(**CASES[k]["universe"]) for k in names]
    with ug.Packer(us, precision=precision, rounds_per_sync=8, use_graph=True) as p:
        p.run()
        bad = []
        for k, name in enumerate(names):
            st = p.stats(k)
            idx, gid = p.accepted(k)
            try:
                _check(name, st, idx, gid)
            except AssertionError as e:
                bad.append(str(e))
    assert not bad, f"{len(bad)} of 256 universes differ: " + "; ".join(bad[:4])


def test_c3_sample_single_universe_fp64(ug):
    """The plain FP64 single-universe form (one universe per packer) on a sample of c3
    that holds every 3+1 universe with F >= 200 and the largest caps."""
    names = [k for k in CASES if k.startswith("c3/")]
    big = [k for k in names if CASES[k]["universe"]["dim"] == 3 and CASES[k]["universe"]["T"] >= 200]
    caps = sorted(names, key=lambda k: -CASES[k]["universe"]["attempts"])[:6]
    for name in dict.fromkeys(big + caps):
        u = ug.Universe(**CASES[name]["universe"])
        with ug.Packer([u], precision=0) as p:
            p.run()
            idx, gid = p.accepted(0)
            _check(name, p.stats(0), idx, gid)
