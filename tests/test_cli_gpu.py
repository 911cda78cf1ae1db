"""Drop-in executables end to end on the GPU: braid_knot against the reference
binary's own dump (fixture), braid_cuda through braidlab.engine."""

import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "universe-generator_b200", "bin")


def _run(exe, args):
    return subprocess.run([sys.executable, os.path.join(BIN, exe), *args], capture_output=True,
                          text=True, timeout=600)


def test_braid_knot_executable_reproduces_reference_dump(tmp_path, oracle):
    gold = json.load(open(os.path.join(ROOT, "tests", "golden", "braid_knot_b200.json")))
    r0 = gold["runs"][0]
    dump = tmp_path / "k.csv"
    args = ["-t", str(r0["T"]), "--dim", str(r0["dim"]), "--seed", str(r0["seed"]),
            "--attempts", str(r0["attempts"]), "--dump", str(dump)]
    r = _run("braid_knot", args)
    assert r.returncode == 0, r.stderr
    assert f"done: N={len(r0['idx'])} " in r.stderr
    rows = oracle.parse_knot_dump(dump.read_text(), r0["dim"], r0["T"] - 1)
    assert [x["idx"] for x in rows] == r0["idx"]
    ref_rows = oracle.parse_knot_dump("\n".join(r0["head_rows"]), r0["dim"], r0["T"] - 1)
    for a, b in zip(rows, ref_rows):
        assert np.array_equal(a["b"], b["b"])
        np.testing.assert_allclose(a["a"], b["a"], rtol=1e-14)
        np.testing.assert_allclose(a["f"], b["f"], rtol=1e-14)


def test_braid_cuda_through_braidlab_engine(tmp_path, oracle):
    from braidlab.config import Job
    from braidlab.engine import binary_name, build_command, parse_done
    from ugb200.io import load_dump

    job = Job(dim=2, t=16, seed=5, accept_rate=1e-9, max_attempts=30000.0)
    curve = tmp_path / "c.csv"
    cmd = build_command(job, binary_name(job.dim, job.terms), str(curve))
    dump = tmp_path / "d.csv"
    r = _run(cmd[0], cmd[1:] + ["--dump-params", str(dump)])
    assert r.returncode == 0, r.stderr
    n, att = parse_done(r.stderr)
    ref = oracle.pack(oracle.Model(dim=2, T=16, terms=2, rng=oracle.RNG_KNOT, seed=5), 30000)
    assert (n, att) == (len(ref.acc_idx), 30000)
    lines = curve.read_text().splitlines()
    assert lines[0] == "attempts,n" and lines[-1] == f"30000,{n}"
    dim, a2, a, b, f, gid = load_dump(dump)
    assert dim == 2 and a.shape == (n, 2, 1) and gid is None
    c = oracle.candidate(oracle.Model(dim=2, T=16, terms=2, rng=oracle.RNG_KNOT, seed=5),
                         int(ref.acc_idx[-1]))
    np.testing.assert_allclose(a[-1], c["a"], rtol=1e-9)  # %.10g in the dump


def test_braid_cuda_subpaths_curve_columns(tmp_path):
    curve = tmp_path / "c.csv"
    r = _run("braid_cuda", ["-t", "12", "--seed", "4", "--attempts", "3000", "--terms", "12",
                            "--subpaths", "--sub-attempts", "20000", "--curve", str(curve)])
    assert r.returncode == 0, r.stderr
    lines = curve.read_text().splitlines()
    assert lines[0] == "attempts,n,nsub,filled"
    last = [int(v) for v in lines[-1].split(",")]
    assert last[0] == 23000 and last[2] > 0 and last[3] > 0
    # the done lines carry the occupied cells as braid_cuda.cu:945 and :1039-1042 print them
    assert ", filled " in r.stderr and "sub done (attempt budget): Nsub=" in r.stderr
    assert f"filled {last[3]}/" in r.stderr.split("sub done")[1]


def test_braid_cuda_sub_until_fill_rate(tmp_path):
    """--sub-until-fill-rate stops phase 2 on the windowed new-volume rate (windows of at
    least 2e7 attempts, after 1e6 phase-2 attempts, braid_cuda.cu:1024-1035)."""
    r = _run("braid_cuda", ["-t", "24", "--excl", "open", "--zgrid", "mid", "--seed", "4",
                            "--attempts", "20000", "--terms", "24", "--subpaths",
                            "--sub-attempts", "60000000", "--sub-until-fill-rate", "5e-4"])
    assert r.returncode == 0, r.stderr
    assert "sub done (fill-rate): Nsub=" in r.stderr
    sub_att = int(r.stderr.split("sub done (fill-rate): Nsub=")[1].split(" in ")[1].split()[0])
    assert 20_000_000 <= sub_att < 60_000_000


def test_braid_cuda3d_euclid_collision(tmp_path, oracle):
    r = _run("braid_cuda3d", ["-t", "16", "--seed", "3", "--attempts", "20000", "--terms", "16",
                              "--euclid-collision", "--rng", "philox"])
    assert r.returncode == 0, r.stderr
    ref = oracle.pack(oracle.Model(dim=3, T=16, seed=3, euclid=1), 20000)
    assert f"done: N={len(ref.acc_idx)} in 20000 attempts" in r.stderr


def test_braid_cuda3d_diag_probe(tmp_path, oracle):
    """--diag: occupancy histogram of the accepted x over all timesteps and the probe of
    fresh proposals against the final packing (braid_cuda3d.cu:1615-1670)."""
    pre = tmp_path / "d"
    r = _run("braid_cuda3d", ["-t", "12", "--seed", "2", "--attempts", "20000", "--terms", "12",
                              "--rng", "philox", "--diag", str(pre), "--probe-n", "20000"])
    assert r.returncode == 0, r.stderr
    assert f"diag: wrote {pre}_occ.csv and {pre}_probe.csv (probeN=20000)" in r.stderr
    occ = np.loadtxt(f"{pre}_occ.csv", delimiter=",", skiprows=1)
    prb = np.loadtxt(f"{pre}_probe.csv", delimiter=",", skiprows=1)
    n = len(oracle.pack(oracle.Model(dim=3, T=12, seed=2), 20000).acc_idx)
    assert occ.shape == (50, 2) and int(occ[:, 1].sum()) == n * 12
    assert int(prb[:, 1].sum()) == 20000 and 0 < int(prb[:, 2].sum()) < 20000
    assert np.all(prb[:, 2] <= prb[:, 1])


def test_probe_counts_match_the_oracle(ug, oracle):
    """Probe candidates are the candidates of the stream keyed by the probe seed, tested
    against the packing: the accepted count equals the oracle's test of the same stream."""
    u = ug.Universe(dim=2, T=16, seed=5, attempts=20000, round_size=2048)
    ref = oracle.pack(oracle.Model(dim=2, T=16, seed=5), 20000)
    with ug.Packer([u]) as p:
        p.run()
        prop, acc = p.probe(0, n=1000, bins=50, seed=777)
    probe_m = oracle.Model(dim=2, T=16, seed=777)
    m = oracle.Model(dim=2, T=16, seed=5)
    packed = [oracle.positions(m, int(i)) for i in ref.acc_idx]
    cell = 2.0 / 16
    free = 0
    for i in range(1000):
        P = oracle.positions(probe_m, i)
        hit = False
        for Q in packed:
            d = np.abs(P - Q)
            d = np.minimum(d, 2.0 - d)
            if np.any(np.all(d <= cell, axis=0)):
                hit = True
                break
        free += not hit
    assert int(prop.sum()) == 1000 and int(acc.sum()) == free
