"""The CPU oracle pinned against the reference's own code and published vectors.

Golden data: tests/golden/knot_reference.json, made by tests/golden/make_golden.py
from the reference's cuda/braid_knot.cu (compiled unmodified, run on the CPU).
"""

import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden", "knot_reference.json")


def _parse(row: str, dim: int, nw: int):
    v = row.split(",")
    k = 2
    out = {"idx": int(v[1]) - 1, "a2": [], "b": [], "a": [], "f": []}
    for _ in range(dim):
        out["a2"].append(float(v[k])); k += 1
        bb, aa, ff = [], [], []
        for _ in range(nw):
            bb.append(int(v[k])); aa.append(float(v[k + 1])); ff.append(float(v[k + 2])); k += 3
        out["b"].append(bb); out["a"].append(aa); out["f"].append(ff)
    return out


def _model(O, c):
    return O.Model(dim=c["dim"], T=c["T"], terms=c["terms"], rng=O.RNG_KNOT,
                   pin=c["pin"], seed=c["seed"])


def test_philox_published_vectors(oracle):
    # Random123 known-answer vectors for Philox4x32-10 (Salmon et al., SC'11)
    assert [hex(x) for x in oracle.philox([0, 0, 0, 0], [0, 0])] == \
        ["0x6627e8d5", "0xe169c58d", "0xbc57ac4c", "0x9b00dbd8"]
    assert [hex(x) for x in oracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)] == \
        ["0x408f276d", "0x41c83b0e", "0xa20bc7c6", "0x6d5451fd"]
    assert [hex(x) for x in oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                                          [0xA4093822, 0x299F31D0])] == \
        ["0xd16cfe09", "0x94fdcceb", "0x5001e420", "0x24126ea1"]


def test_knot_stream_matches_reference():
    import oracle as O
    gold = json.load(open(GOLD))
    for s in gold["streams"]:
        m = _model(O, s)
        for row in s["rows"]:
            r = _parse(row, s["dim"], m.nw)
            c = O.candidate(m, r["idx"])
            assert np.array_equal(c["b"], np.array(r["b"]))
            assert np.array_equal(c["a"], np.array(r["a"]))  # bit-exact (%.17g round trip)
            assert np.array_equal(c["f"], np.array(r["f"]))
            assert np.array_equal(c["a2"], np.array(r["a2"]))


def test_knot_packing_matches_reference():
    import oracle as O
    gold = json.load(open(GOLD))
    for p in gold["packs"]:
        m = _model(O, p)
        res = O.pack(m, p["attempts"])
        assert list(res.acc_idx) == p["idx"], p
        assert f"done: N={len(res.acc_idx)} in {res.attempts} attempts" == p["done"]
        for row in p["head_rows"] + p["tail_rows"]:
            r = _parse(row, p["dim"], m.nw)
            c = O.candidate(m, r["idx"])
            assert np.array_equal(c["a"], np.array(r["a"]))
            assert np.array_equal(c["a2"], np.array(r["a2"]))


def test_live_reference_harness_random_configs():
    """Cross-check against oracle/_ref/knot_host when it is built (reference tree present)."""
    import oracle as O
    if not os.path.exists(os.path.join(O.REF_DIR, "knot_host")):
        pytest.skip("reference harness not built")
    rng = np.random.default_rng(5)
    for _ in range(4):
        dim = int(rng.integers(1, 4)); T = int(rng.integers(6, 20)); seed = int(rng.integers(0, 1 << 40))
        terms = int(rng.choice([0, 3, T]))
        m = O.Model(dim=dim, T=T, terms=terms, rng=O.RNG_KNOT, seed=seed)
        args = ["-t", str(T), "--dim", str(dim), "--seed", str(seed), "--attempts", "3000"]
        if terms:
            args += ["--terms", str(terms)]
        ref = O.parse_knot_dump(O.knot_host(["--mode", "pack"] + args).stdout, dim, m.nw)
        res = O.pack(m, 3000)
        assert [r["idx"] for r in ref] == list(res.acc_idx)


@pytest.mark.parametrize("rng", [0, 1])
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_threaded_form_equals_sequential(oracle, rng, dim):
    m = oracle.Model(dim=dim, T=12, rng=rng, zgrid=dim % 2, excl=(dim + 1) % 2, seed=31 + dim)
    a = oracle.pack(m, 6000)
    b = oracle.pack(m, 6000, nthreads=4, round_size=512)
    assert np.array_equal(a.acc_idx, b.acc_idx)


def _pairwise_ok(P, cell, inclusive, cross=False):
    """No two accepted trajectories violate the exclusion at any timestep."""
    n = len(P)
    for i in range(n):
        d = P[i][None] - P[:i]
        d = np.where(d > 1, d - 2, np.where(d < -1, d + 2, d))
        ad = np.abs(d)
        hit = (ad <= cell) if inclusive else (ad < cell)
        if hit.all(axis=1).any(axis=-1).any():
            return False
        if cross:
            s = d[:, 0, :]
            flip = ((s[:, :-1] < 0) != (s[:, 1:] < 0)) & (np.abs(s[:, :-1]) + np.abs(s[:, 1:]) < 1)
            if flip.any():
                return False
    return True


@pytest.mark.parametrize("conv", [(0, 0), (1, 1)])
def test_accepted_sets_are_exclusion_free(oracle, conv):
    for dim in (1, 2, 3):
        m = oracle.Model(dim=dim, T=16, zgrid=conv[0], excl=conv[1], seed=dim,
                         cross1d=int(dim == 1 and conv[1] == 1))
        res = oracle.pack(m, 8000)
        P = np.stack([oracle.positions(m, int(i)) for i in res.acc_idx])
        cell = 2 / 16 if conv[1] == 0 else 1 / 16
        assert _pairwise_ok(P, cell, conv[1] == 0, cross=bool(m.cross1d))


def test_budget_and_phase_rules(oracle):
    """sum_b b|a_b| = 1 per axis, phases only on even b, a2 in [-1, 1)."""
    for rng in (0, 1):
        m = oracle.Model(dim=3, T=32, rng=rng, seed=9)
        for idx in (0, 1, 12345):
            c = oracle.candidate(m, idx)
            for ax in range(3):
                assert abs(np.sum(np.abs(c["a"][ax]) * c["b"][ax]) - 1.0) < 1e-12
                odd = c["b"][ax] % 2 == 1
                assert np.all(c["f"][ax][odd] == 0)
                assert np.all((c["f"][ax] >= 0) & (c["f"][ax] < np.pi))
                assert sorted(c["b"][ax]) == list(range(2, 33))
            assert np.all((c["a2"] >= -1) & (c["a2"] < 1))


def test_group_modes(oracle):
    m = oracle.Model(dim=2, T=12, seed=4)
    r = oracle.pack(m, 3000, group_mode=oracle.GROUP_SUBPATH, sub_attempts=20000)
    assert r.n_sub > 0 and r.n_unique + r.n_sub == len(r.acc_idx)
    uniq = r.gid[: r.n_unique]
    assert np.array_equal(uniq, np.arange(r.n_unique))
    assert np.all(r.acc_idx[r.n_unique:] >= r.phase1_end)
    assert np.all(r.gid[r.n_unique:] < r.n_unique)
    u = oracle.pack(m, 20000, group_mode=oracle.GROUP_UNIQUE)
    founders = np.flatnonzero(u.gid == np.arange(len(u.gid)))
    assert len(founders) == u.n_unique and u.n_sub == len(u.gid) - u.n_unique


def test_oracle_matches_reference_gpu_binary():
    """Accepted sets of the reference's own GPU packer (braid_knot run on a B200)."""
    import oracle as O
    gold = json.load(open(os.path.join(os.path.dirname(GOLD), "braid_knot_b200.json")))
    for r in gold["runs"]:
        m = O.Model(dim=r["dim"], T=r["T"], rng=O.RNG_KNOT, pin=r["pin"], seed=r["seed"])
        res = O.pack(m, r["attempts"])
        assert list(res.acc_idx) == r["idx"], r["command"]
        for row in r["head_rows"]:
            p = _parse(row, r["dim"], m.nw)
            c = O.candidate(m, p["idx"])
            assert np.array_equal(c["a"], np.array(p["a"])) and np.array_equal(c["f"], np.array(p["f"]))


@pytest.mark.parametrize("dim,excl", [(2, 0), (3, 1), (2, 1)])
def test_euclid_exclusion_against_brute_force(oracle, dim, excl):
    """The L2-ball exclusion (--euclid-collision, cuda/braid_cuda3d.cu:605-608) of the
    oracle against sequential RSA written out pairwise over all timesteps; both the
    threaded batch form and the plain sequential form."""
    m = oracle.Model(dim=dim, T=10, zgrid=1, excl=excl, seed=17 + dim, euclid=1)
    n = 400
    pos = np.stack([oracle.positions(m, i) for i in range(n)])  # [n][dim][T]
    cell = 2.0 / 10 if excl == 0 else 1.0 / 10
    acc = []
    for i in range(n):
        ok = True
        for j in acc:
            d = pos[i] - pos[j]
            d = np.where(d > 1.0, d - 2.0, np.where(d < -1.0, d + 2.0, d))
            s = np.zeros(d.shape[1])
            for ax in range(dim):
                s = s + d[ax] * d[ax]
            if np.any(s <= cell * cell if excl == 0 else s < cell * cell):
                ok = False
                break
        if ok:
            acc.append(i)
    for nth in (1, 4):
        res = oracle.pack(m, n, nthreads=nth, round_size=64)
        assert res.acc_idx.tolist() == acc
    cheb = oracle.pack(oracle.Model(dim=dim, T=10, zgrid=1, excl=excl, seed=17 + dim), n)
    assert len(acc) > len(cheb.acc_idx)  # the ball excludes less than the cube


def _win_stop(idx, start, budget, thr):
    """The windowed stop restated in numpy: buckets of q = clamp(30/thr, 2e7, 5e9) // 32
    candidates from the phase start; at each boundary b (phase-relative) with 32
    buckets behind it and b > 1e6, stop when admissions in the last 32 q / (32 q) < thr."""
    W = int(min(5e9, max(2e7, 30.0 / thr)))
    q = max(1, W // 32)
    rel = np.sort(np.asarray(idx, np.int64) - start)
    for j in range(32, budget // q + 1):
        b = j * q
        cnt = np.searchsorted(rel, b) - np.searchsorted(rel, b - 32 * q)
        if b > 1_000_000 and cnt / (32 * q) < thr:
            return start + b
    return start + budget


def test_accept_rate_window_stop(oracle):
    """--until-accept-rate (braid_cuda.cu:931-943) with candidate-aligned buckets: the
    stop lands on the first bucket boundary where the rule holds, and the run equals a
    budget-limited run to the same attempt count."""
    m = oracle.Model(dim=2, T=8, zgrid=1, excl=1, seed=21)
    full = oracle.pack(m, 40_000_000, nthreads=8, round_size=65536, accept_rate=1e-6)
    assert 20_000_000 < full.attempts < 40_000_000  # not at the first full window
    assert full.attempts == _win_stop(full.acc_idx, 0, 40_000_000, 1e-6)
    cut = oracle.pack(m, full.attempts, nthreads=8, round_size=65536)
    assert np.array_equal(cut.acc_idx, full.acc_idx)
