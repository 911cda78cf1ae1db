"""Observer-view remap (braidlab/frames.py:147-188) and the per-frame measurements
beside it, on the CPU: the oracle against the reference's own outputs, the mirror's
measurements, and the C ABI's argument checks (no device work).

Golden data: tests/golden/view_reference.json, made by tests/golden/make_view_golden.py."""

import ctypes
import json
import os
import subprocess
import sys

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden", "view_reference.json")
from oracle import REFERENCE_DIR as REF  # noqa: E402


def test_oracle_matches_reference_golden(oracle):
    cases = json.load(open(GOLD))
    assert len(cases) >= 16
    for c in cases:
        ax, ay, ld = oracle.apparent_positions(c["dx"], c["dy"], c["chi"], c["beta"], c["mode"], c["cheb"])
        # the same numpy operations in the same order: equal to the last bit
        np.testing.assert_array_equal(ax, c["ax"])
        np.testing.assert_array_equal(ay, c["ay"])
        np.testing.assert_array_equal(ld, c["ln_dopp"])


def test_golden_covers_the_edge_cases():
    cases = json.load(open(GOLD))
    mags = {round(float(np.hypot(*c["beta"])), 7) for c in cases if c["mode"] == "moving"}
    assert any(m > 0.995 for m in mags) and any(m <= 1e-6 for m in mags)
    assert {c["cheb"] for c in cases} == {True, False} and {c["mode"] for c in cases} == {"static", "moving"}
    for c in cases:  # a hit at the pulse centre keeps its offsets
        assert c["dx"][0] == 0.0 and c["ax"][0] == 0.0 and c["ln_dopp"][0] == 0.0


def _frame(n=40, seed=3):
    from braidlab.frames import HIT_DTYPE, ObserverFrame

    rng = np.random.default_rng(seed)
    h = np.zeros(n, HIT_DTYPE)
    h["src"] = rng.integers(0, 7, n)
    h["dx"] = rng.normal(size=n)
    h["dy"] = rng.normal(size=n)
    h["chi"] = rng.uniform(0.1, 2, n)
    h["z_emit"] = rng.uniform(0.2, 1.2, n)
    return ObserverFrame(1.4, 2.0, 1, 0.1, 0.2, np.array([0.2, 0.1]), np.sort(h, order=["chi", "src"]))


def test_mirror_measurements(tmp_path):
    from braidlab.frames import counts_vs_redshift, ghost_multiplicity, load_gids

    fr = _frame()
    edges = np.linspace(1.0, 3.0, 9)
    hist, cum = counts_vs_redshift(fr, edges)
    z = np.sin(1.4) / np.sin(fr.hits["z_emit"].astype(np.float64))
    assert hist.sum() == np.count_nonzero((z >= 1.0) & (z <= 3.0)) and cum[-1] == hist.sum()
    assert np.array_equal(ghost_multiplicity(fr), np.bincount(fr.hits["src"]))
    p = tmp_path / "d.csv"
    p.write_text("a,b,gid\n1,2,0\n3,4,0\n5,6,2\n")
    assert load_gids(p).tolist() == [0, 0, 2]
    q = tmp_path / "e.csv"
    q.write_text("a,b\n1,2\n")
    with pytest.raises(ValueError):
        load_gids(q)


def test_mirror_measurements_match_reference(tmp_path):
    if not os.path.isdir(os.path.join(REF, "braidlab")):
        pytest.skip("reference tree not present")
    from braidlab.frames import counts_vs_redshift, ghost_multiplicity

    fr = _frame(60, 5)
    np.save(tmp_path / "h.npy", fr.hits)
    code = ("import sys, json; sys.path.insert(0, sys.argv[1]); import numpy as np;"
            "from braidlab.frames import ObserverFrame, counts_vs_redshift, ghost_multiplicity;"
            "h = np.load(sys.argv[2]); fr = ObserverFrame(1.4, 2.0, 1, 0.1, 0.2, np.array([0.2, 0.1]), h);"
            "a, b = counts_vs_redshift(fr, np.linspace(1.0, 3.0, 9));"
            "print(json.dumps([a.tolist(), b.tolist(), ghost_multiplicity(fr).tolist()]))")
    r = subprocess.run([sys.executable, "-c", code, REF, str(tmp_path / "h.npy")], capture_output=True,
                       text=True, check=True)
    ref = json.loads(r.stdout)
    a, b = counts_vs_redshift(fr, np.linspace(1.0, 3.0, 9))
    assert [a.tolist(), b.tolist(), ghost_multiplicity(fr).tolist()] == ref


def test_abi_rejects_a_bad_mode_before_device_work(ug):
    from ugb200 import _lib

    lib = _lib.load()
    out = np.zeros(3)
    h = np.zeros(1, dtype=[("src", "<u4"), ("dx", "<f4"), ("dy", "<f4"), ("chi", "<f4"), ("z_emit", "<f4")])
    rc = lib.ug_apparent_positions(h.ctypes.data, 1, 0.1, 0.0, 7, 1, out.ctypes.data, out.ctypes.data,
                                   out.ctypes.data)
    assert rc == 1 and "static|moving" in _lib.last_error()
    assert lib.ug_apparent_positions(None, 0, 0.1, 0.0, 1, 1, None, None, None) == 0  # nothing to do
    assert lib.ug_apparent_positions(None, -1, 0.1, 0.0, 1, 1, None, None, None) == 1
    with pytest.raises(ValueError):
        from ugb200.frames import apparent_positions

        apparent_positions(h, (0.1, 0.0), "sideways")


@pytest.mark.parametrize("cheb", [True, False])
def test_oracle_remap_properties(oracle, cheb):
    """Images stay on their own shell, centre hits stay put, boosts above the cap act
    as the cap, boosts under 1e-6 and the static mode return the stored offsets."""
    rng = np.random.default_rng(7)
    n = 1 << 14
    chi = rng.uniform(1e-3, 4.0, n).astype(np.float32)
    ang = rng.uniform(-np.pi, np.pi, n)
    dx = (chi * np.cos(ang)).astype(np.float32)
    dy = (chi * np.sin(ang)).astype(np.float32)
    dx[::101] = 0.0
    dy[::101] = 0.0
    moved = (dx != 0) | (dy != 0)
    ax, ay, ld = oracle.apparent_positions(dx, dy, chi, (0.5, -0.6), "moving", cheb)
    r = np.maximum(np.abs(ax), np.abs(ay)) if cheb else np.hypot(ax, ay)
    np.testing.assert_allclose(r[moved], chi[moved].astype(np.float64), rtol=1e-12)
    assert np.all(ax[~moved] == 0) and np.all(ld[~moved] == 0)
    cap = oracle.apparent_positions(dx, dy, chi, (0.995 * 0.6, 0.995 * 0.8), "moving", cheb)
    over = oracle.apparent_positions(dx, dy, chi, (6.0, 8.0), "moving", cheb)
    for a, b in zip(cap, over):
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)
    for beta, mode in (((3e-7, 4e-7), "moving"), ((0.5, 0.5), "static")):
        sx, sy, sl = oracle.apparent_positions(dx, dy, chi, beta, mode, cheb)
        assert np.array_equal(sx, dx.astype(np.float64)) and np.array_equal(sy, dy.astype(np.float64))
        assert not sl.any()
