"""Checkpoint / resume of a run: a universe stopped after some rounds, saved (admissions
+ state block), rebuilt in another packer and run on admits exactly what the
uninterrupted run admits, with the same counters."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    dict(dim=2, T=32, zgrid=1, excl=1, seed=3, attempts=200000, round_size=4096),              # dense grid
    dict(dim=3, T=48, zgrid=1, excl=1, seed=5, attempts=60000, round_size=4096),               # 3+1
    dict(dim=2, T=16, seed=7, attempts=4000, group_mode=1, sub_attempts=60000, round_size=1024),  # across phases
    dict(dim=2, T=24, zgrid=1, excl=1, seed=8, attempts=60000, group_mode=2, round_size=2048),  # unique groups
    dict(dim=2, T=16, rng=1, seed=2, attempts=50000, round_size=2048),                          # knot stream
    dict(dim=1, T=20, zgrid=1, excl=1, cross1d=1, seed=4, attempts=40000, round_size=2048),    # 1+1D crossing
]


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("precision", [0, 1])
def test_resume_equals_uninterrupted(ug, case, precision, tmp_path):
    u = ug.Universe(**CASES[case])
    with ug.Packer([u], precision=precision) as p:
        p.run()
        full = p.stats(0)
        a, g = p.accepted(0)
    with ug.Packer([u], precision=precision, rounds_per_sync=1) as p:
        p.run(max_rounds=3)
        mid = p.stats(0)
        ck = p.checkpoint(0)
    assert 0 < mid.attempts < full.attempts
    ug.save_checkpoint(tmp_path / "ck.npz", ck)
    ck2 = ug.load_checkpoint(tmp_path / "ck.npz")
    # resume in a different batch (another universe in front), other precision
    other = ug.Universe(dim=2, T=16, seed=99, attempts=5000, round_size=1024)
    with ug.Packer([other, u], precision=1 - precision, force_hash=bool(case % 2)) as q:
        q.restore(1, ck2)
        r0 = q.stats(1)
        assert (r0.n, r0.attempts, r0.filled) == (mid.n, mid.attempts, mid.filled)
        q.run()
        st = q.stats(1)
        b, h = q.accepted(1)
    assert np.array_equal(a, b) and np.array_equal(g, h)
    assert (st.n, st.n_unique, st.n_sub, st.attempts, st.phase1_end, st.filled) == \
        (full.n, full.n_unique, full.n_sub, full.attempts, full.phase1_end, full.filled)


def test_restore_rejects_a_foreign_state(ug):
    u = ug.Universe(dim=2, T=16, seed=1, attempts=20000, round_size=2048)
    with ug.Packer([u]) as p:
        p.run(max_rounds=2)
        ck = p.checkpoint(0)
    v = ug.Universe(dim=2, T=16, seed=2, attempts=20000, round_size=2048)
    with ug.Packer([v]) as q:
        with pytest.raises(ug.UgError):
            q.restore(0, ck)
        bad = dict(ck, idx=ck["idx"][:-1], gid=ck["gid"][:-1])
        with pytest.raises(ug.UgError):
            ug.Packer([u]).restore(0, bad)
