"""The braidlab call surface (engine / config), the engine-compatible command
line and the dump/curve formats, checked on the CPU.

Where the reference tree is present, the mirror is compared with the reference's
own braidlab in a subprocess (the two packages share a name)."""

import json
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import REFERENCE_DIR as REF  # noqa: E402
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "universe-generator_b200")

JOBS = [dict(dim=d, t=t, seed=s, accept_rate=r, max_attempts=m, terms=k, subpaths=sp,
             sub_attempts=sa, euclid=eu, sparse=spr, tag=tag)
        for d, t, s, r, m, k, sp, sa, eu, spr, tag in [
            (2, 44, 2, 1e-7, 3e12, 2, False, 0, False, False, ""),
            (3, 44, 2, 1e-6, 3e12, 10, False, 0, False, False, "fqe6"),
            (2, 120, 7, 1e-6, 2e9, 2, True, 0, False, False, ""),
            (2, 60, 1, 1e-5, 1e8, 60, True, 5e8, False, False, "e5"),
            (3, 200, 3, 1e-7, 3e12, 2, False, 0, True, True, ""),
            (3, 360, 9, 1e-6, 3e12, 360, False, 0, False, True, "x"),
        ]]

SCRIPT = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
from braidlab.config import Job, Campaign
from braidlab.engine import build_command, parse_done, binary_name
jobs = json.loads(sys.argv[2])
out = {"cmd": [], "name": [], "key": [], "bin": [], "done": [], "camp": []}
for j in jobs:
    J = Job(**j)
    out["cmd"].append(build_command(J, "bin", "c.csv"))
    out["name"].append(J.name); out["key"].append(list(J.key))
for d in (2, 3):
    for k in (2, 10, 11, 150):
        out["bin"].append(binary_name(d, k))
for s in ["done: N=12 in 3400 attempts", "x\ndone:  N=5  in 7 attempts, filled 1/2", "nope"]:
    out["done"].append(parse_done(s))
c = Campaign(name="c", dim=2, t_values=(20, 40), seeds=(1, 2), accept_rate=1e-6,
             terms_values=(2, 5), subpaths=True, sub_attempts=1e6, tag="t")
out["camp"] = [[j.name, list(j.key), j.terms, j.sub_attempts] for j in c.jobs()]
c2 = Campaign(name="c2", dim=3, t_values=(16, 32), seeds=(3,), accept_rate=1e-7, terms_track_t=True)
out["camp"] += [[j.name, list(j.key), j.terms, j.sub_attempts] for j in c2.jobs()]
print(json.dumps(out))
"""


def _surface(root: str) -> dict:
    r = subprocess.run([sys.executable, "-c", SCRIPT, root, json.dumps(JOBS)],
                       capture_output=True, text=True, check=True)
    return json.loads(r.stdout)


def test_mirror_matches_reference_braidlab():
    if not os.path.isdir(os.path.join(REF, "braidlab")):
        pytest.skip("reference tree not present")
    assert _surface(PKG) == _surface(REF)


def test_mirror_identities():
    from braidlab.config import Campaign, Job
    from braidlab.engine import binary_name, build_command, parse_done

    j = Job(dim=3, t=44, seed=2, accept_rate=1e-7, max_attempts=3e12)
    assert j.name == "d3_nyq_T44_s2_ph" and j.key == (3, "nyq", 44, 2, 1e-7, 2)
    cmd = build_command(j, "bin", "curve.csv")
    assert cmd[cmd.index("--maxfreq") + 1] == "44" and cmd[-2:] == ["--curve", "curve.csv"]
    assert {"--uniform", "--torus", "--phase"} <= set(cmd)
    assert binary_name(2, 11) == "braid_cuda_w150" and binary_name(3, 2) == "braid_cuda3d"
    assert parse_done("done: N=3 in 99 attempts") == (3, 99)
    with pytest.raises(ValueError):
        Job(dim=3, t=44, seed=2, accept_rate=1e-7, max_attempts=3e12, band="safe")
    with pytest.raises(ValueError):
        Job(dim=3, t=44, seed=2, accept_rate=1e-7, max_attempts=3e12, subpaths=True)
    with pytest.raises(ValueError):
        Campaign(name="c", dim=2, t_values=(4,), seeds=(1,), accept_rate=1e-6,
                 terms_values=(3,), terms_track_t=True)


@pytest.mark.parametrize("argv,msg", [
    (["--smart"], "--smart"), (["-t", "16", "--maxfreq", "12"], "maxfreq"),
    (["--bogus"], "unknown flag"), (["--euclid-collision"], "L2"),
    (["--nu-attempts", "10"], "nu"), (["-t"], "needs a value"),
])
def test_cli_rejects_bad_flags_before_any_device_work(argv, msg):
    r = subprocess.run([sys.executable, os.path.join(PKG, "bin", "braid_cuda"), *argv],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "error:" in r.stderr and msg in r.stderr


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("nw", [1, 4])
def test_dump_round_trip(tmp_path, dim, nw):
    from ugb200.io import load_dump, write_dump

    rng = np.random.default_rng(dim * 10 + nw)
    n = 5
    a2 = rng.uniform(-1, 1, (n, dim))
    a = rng.normal(0, 0.1, (n, dim, nw))
    b = rng.integers(2, 30, (n, dim, nw))
    f = np.where(b % 2 == 0, rng.uniform(0, np.pi, (n, dim, nw)), 0.0)
    gid = np.arange(n)
    p = tmp_path / "d.csv"
    write_dump(p, dim, a2, a, b, f, gid=gid)
    d2, A2, A, B, Fh, G = load_dump(p)
    assert d2 == dim and np.array_equal(G, gid) and np.array_equal(B, b)
    np.testing.assert_allclose(A, a, rtol=1e-9)
    np.testing.assert_allclose(A2, a2, rtol=1e-9)
    np.testing.assert_allclose(Fh, f, rtol=1e-9, atol=1e-12)


def test_dump_layout_matches_reference_readers(tmp_path):
    """The reference's own dump reader (corrdim.load_axis_terms) reads our dumps."""
    if not os.path.isdir(os.path.join(REF, "braidlab")):
        pytest.skip("reference tree not present")
    from ugb200.io import write_dump

    rng = np.random.default_rng(3)
    for dim, nw in [(2, 1), (2, 5), (3, 1), (3, 5)]:
        a2 = rng.uniform(-1, 1, (4, dim)); a = rng.normal(0, 0.1, (4, dim, nw))
        b = rng.integers(2, 30, (4, dim, nw)); f = rng.uniform(0, 3, (4, dim, nw))
        p = tmp_path / f"d{dim}{nw}.csv"
        write_dump(p, dim, a2, a, b, f)
        code = ("import sys, json; sys.path.insert(0, sys.argv[1]);"
                "from braidlab.corrdim import load_axis_terms;"
                "ax = load_axis_terms(sys.argv[2]);"
                "print(json.dumps([[x.a.tolist(), x.b.tolist(), x.f.tolist(), x.a2.tolist()] for x in ax]))")
        r = subprocess.run([sys.executable, "-c", code, REF, str(p)], capture_output=True,
                           text=True, check=True)
        got = json.loads(r.stdout)
        assert len(got) == dim
        for k in range(dim):
            np.testing.assert_allclose(np.array(got[k][0]), a[:, k, :], rtol=1e-9)
            np.testing.assert_allclose(np.array(got[k][1]), b[:, k, :])
            np.testing.assert_allclose(np.array(got[k][3]), a2[:, k], rtol=1e-9)


def test_curve_rows_are_exact_milestones():
    from ugb200.io import curve_rows, milestones

    acc = np.array([0, 1, 5, 999, 1000, 1200, 5000])
    rows = curve_rows(acc, 6000)
    ms = milestones(6000)
    assert [r[0] for r in rows] == ms + [6000]
    assert rows[0] == (1000, 4) and rows[-1] == (6000, 7)


def test_brf1_writer_matches_reference_reader(tmp_path):
    """A BRF1 file from ugb200.frames.write_brf1 reads back through the reference's
    own braidlab.frames.load_frames (subprocess; the packages share a name)."""
    from ugb200.frames import HIT_DTYPE, Baked, write_brf1

    rng = np.random.default_rng(1)
    hits = []
    for fi in range(2):
        row = []
        for o in range(2):
            h = np.zeros(5 + fi + o, HIT_DTYPE)
            h["src"] = rng.integers(0, 9, len(h)); h["dx"] = rng.normal(size=len(h))
            h["dy"] = rng.normal(size=len(h)); h["chi"] = rng.uniform(0, 1, len(h))
            h["z_emit"] = rng.uniform(0.1, 1, len(h))
            row.append(h)
        hits.append(row)
    bk = Baked("fit", True, 0.33, 0.0628, -1, [(0, 3, 0.0, 0.0), (1, -1, 0.1, 0.2)],
               np.array([[1.0, 0.9, 3], [1.2, 1.1, 3]]), rng.normal(size=(2, 2, 4)), hits, None, 9)
    p = tmp_path / "f.frames"
    write_brf1(p, bk)
    from braidlab.frames import load_frames
    ours = load_frames(p)
    assert ours.n_paths == 9 and ours.observers[1] == (1, -1, 0.1, 0.2)
    if not os.path.isdir(os.path.join(REF, "braidlab")):
        return
    code = ("import sys, json; sys.path.insert(0, sys.argv[1]);"
            "from braidlab.frames import load_frames; fs = load_frames(sys.argv[2]);"
            "print(json.dumps([fs.n_paths, fs.front, fs.cheb, [list(o) for o in fs.observers],"
            "[[[fr.z_obs, fr.chi_max, fr.wraps, fr.ox, fr.oy, fr.beta.tolist(), fr.hits['chi'].tolist(), fr.hits['src'].tolist()]"
            " for fr in row] for row in fs.frames]]))")
    r = subprocess.run([sys.executable, "-c", code, REF, str(p)], capture_output=True, text=True,
                       check=True)
    ref = json.loads(r.stdout)
    assert ref[0] == 9 and ref[1] == "fit" and ref[2] is True
    for fi, row in enumerate(ref[4]):
        for o, fr in enumerate(row):
            mine = ours.frames[fi][o]
            assert fr[0] == mine.z_obs and fr[2] == mine.wraps
            assert fr[6] == mine.hits["chi"].tolist() and fr[7] == mine.hits["src"].tolist()
