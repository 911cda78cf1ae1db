"""GPU parity: the packer's accepted sets against the CPU oracle (exact),
trajectories and parameters within FP64 tolerance."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

POS_TOL = 1e-12   # FP64: device libm vs host libm, fma vs separate mul/add
PAR_TOL = 1e-14


def _model(O, u):
    return O.Model(dim=u.dim, T=u.T, terms=u.terms, rng=u.rng, zgrid=u.zgrid, excl=u.excl,
                   cross1d=u.cross1d, pin=u.pin_sin1, seed=u.seed, euclid=u.euclid)


def _check(ug, O, u, precision=0, **kw):
    res = O.pack(_model(O, u), u.attempts, max_n=u.max_n, group_mode=u.group_mode,
                 sub_attempts=u.sub_attempts)
    with ug.Packer([u], precision=precision, **kw) as p:
        p.run()
        st = p.stats(0)
        idx, gid = p.accepted(0)
        assert st.done
        assert np.array_equal(idx, res.acc_idx), (len(idx), len(res.acc_idx))
        assert st.attempts == res.attempts
        if u.group_mode:
            assert np.array_equal(gid, res.gid)
            assert (st.n_unique, st.n_sub) == (res.n_unique, res.n_sub)
        pos = p.positions(0)
        m = _model(O, u)
        for k in range(0, len(idx), max(1, len(idx) // 16)):
            ref = O.positions(m, int(idx[k]))
            dd = np.abs(pos[k] - ref)
            dd = np.minimum(dd, 2 - dd)   # wrapped coordinates
            assert dd.max() < POS_TOL
        par = p.params(0)
        for k in range(0, len(idx), max(1, len(idx) // 8)):
            c = O.candidate(m, int(idx[k]))
            assert np.array_equal(par["b"][k], c["b"])
            np.testing.assert_allclose(par["a"][k], c["a"], rtol=PAR_TOL, atol=1e-300)
            np.testing.assert_allclose(par["f"][k], c["f"], rtol=PAR_TOL, atol=1e-300)
            np.testing.assert_allclose(par["a2"][k], c["a2"], rtol=0, atol=1e-15)
        return st, idx


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("rng", [0, 1])
def test_parity_ref_conventions(ug, oracle, dim, rng):
    u = ug.Universe(dim=dim, T=16, rng=rng, seed=100 + dim, attempts=30000, round_size=4096)
    _check(ug, oracle, u)


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_parity_open_mid_conventions(ug, oracle, dim):
    u = ug.Universe(dim=dim, T=16, zgrid=1, excl=1, cross1d=int(dim == 1), seed=7 * dim,
                    attempts=20000, round_size=2048)
    _check(ug, oracle, u)


def test_parity_reference_golden_knot(ug, oracle):
    """The reference's own deterministic packer stream and accepted set (fixture)."""
    import json
    import os
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "knot_reference.json")))
    for p in gold["packs"]:
        u = ug.Universe(dim=p["dim"], T=p["T"], terms=p["terms"], rng=1, pin_sin1=p["pin"],
                        seed=p["seed"], attempts=p["attempts"], round_size=4096)
        with ug.Packer([u]) as pk:
            pk.run()
            idx, _ = pk.accepted(0)
        assert list(idx) == p["idx"], (p["T"], p["dim"])


def test_round_size_independence(ug, oracle):
    u = ug.Universe(dim=2, T=24, seed=5, attempts=60000, round_size=65536)
    _, a = _check(ug, oracle, u)
    for rs in (128, 1024):
        u2 = ug.Universe(dim=2, T=24, seed=5, attempts=60000, round_size=rs)
        with ug.Packer([u2]) as p:
            p.run()
            b, _ = p.accepted(0)
        assert np.array_equal(a, b)


def test_hash_grid_and_growth(ug, oracle):
    u = ug.Universe(dim=3, T=20, seed=9, attempts=30000, round_size=8192)
    _check(ug, oracle, u, force_hash=True, slot_hint=1024)


def test_graph_and_eager_agree(ug, oracle):
    u = ug.Universe(dim=2, T=16, seed=3, attempts=40000, round_size=1024)
    s1, a = _check(ug, oracle, u, use_graph=True, rounds_per_sync=4)
    s2, b = _check(ug, oracle, u, use_graph=False)
    assert np.array_equal(a, b)


def test_max_n_stop(ug, oracle):
    u = ug.Universe(dim=2, T=16, seed=1, attempts=100000, max_n=20, round_size=2048)
    st, idx = _check(ug, oracle, u)
    assert st.n == 20


@pytest.mark.parametrize("precision", [0, 1])
def test_group_subpath_mode(ug, oracle, precision):
    u = ug.Universe(dim=2, T=12, seed=4, attempts=3000, group_mode=1, sub_attempts=20000,
                    round_size=1024)
    st, _ = _check(ug, oracle, u, precision=precision)
    assert st.n_sub > 0


@pytest.mark.parametrize("precision", [0, 1])
def test_group_unique_mode(ug, oracle, precision):
    u = ug.Universe(dim=2, T=16, zgrid=1, excl=1, seed=8, attempts=20000, group_mode=2,
                    round_size=2048)
    st, _ = _check(ug, oracle, u, precision=precision)
    assert st.n_sub > 0


@pytest.mark.parametrize("dim,T,att,mode", [(2, 256, 60000, 2), (3, 48, 40000, 2), (2, 96, 8000, 1)])
def test_group_modes_tensor_core_path(ug, oracle, dim, T, att, mode):
    """Group rounds through the tensor-core prefilter (certain contacts join or reject,
    guard-band contacts go to the FP64 retest): accepted sets and group labels equal the
    oracle's; the unique-group case at F = 256 is the shape of the c4 workload."""
    u = ug.Universe(dim=dim, T=T, zgrid=1, excl=1, seed=5 + T, attempts=att, group_mode=mode,
                    sub_attempts=4 * att if mode == 1 else 0, round_size=4096)
    st, _ = _check(ug, oracle, u, precision=1)
    assert st.n_sub > 0


def test_batched_universes_match_single(ug, oracle):
    rng = np.random.default_rng(0)
    us = []
    for k in range(12):
        dim = int(rng.integers(1, 4))
        T = int(rng.choice([8, 12, 16, 24]))
        us.append(ug.Universe(dim=dim, T=T, zgrid=1, excl=1, cross1d=int(dim == 1), seed=k,
                              attempts=int(rng.integers(2000, 20000)), round_size=2048))
    with ug.Packer(us) as p:
        p.run()
        for k, u in enumerate(us):
            idx, _ = p.accepted(k)
            ref = oracle.pack(_model(oracle, u), u.attempts)
            assert np.array_equal(idx, ref.acc_idx), k


def test_parity_reference_gpu_binary(ug):
    """Accepted sets of the reference's own GPU packer (braid_knot on a B200, fixture)."""
    import json
    import os
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "braid_knot_b200.json")))
    for r in gold["runs"]:
        u = ug.Universe(dim=r["dim"], T=r["T"], rng=1, pin_sin1=r["pin"], seed=r["seed"],
                        attempts=r["attempts"], round_size=8192)
        with ug.Packer([u]) as pk:
            pk.run()
            idx, _ = pk.accepted(0)
        assert list(idx) == r["idx"], r["command"]


@pytest.mark.parametrize("precision", [0, 1])
def test_round_sizes_stay_within_buffers(ug, oracle, precision):
    """Survivor-capacity steering never grows a round past its buffers
    (T=200: the initial round size is not a power-of-two fraction of the cap)."""
    u = ug.Universe(dim=2, T=200, zgrid=1, excl=1, seed=2, attempts=60000, round_size=16384)
    _check(ug, oracle, u, precision=precision)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("excl,T", [(0, 9), (0, 17), (0, 25), (1, 13), (1, 21)])
def test_seam_blocks_when_cells_are_not_a_multiple_of_eight(ug, oracle, precision, excl, T):
    """Neighbourhoods that wrap across the seam where the last occupancy block is
    short (gw = 9, 17, 25, 26, 42 cells): every block of the range must be checked."""
    for dim in (1, 2, 3):
        for seed in range(3):
            u = ug.Universe(dim=dim, T=T, zgrid=excl, excl=excl, seed=1000 * dim + seed,
                            attempts=6000, round_size=1024)
            ref = oracle.pack(_model(oracle, u), u.attempts)
            with ug.Packer([u], precision=precision) as p:
                p.run()
                idx, _ = p.accepted(0)
            assert np.array_equal(idx, ref.acc_idx), (dim, seed)


@pytest.mark.parametrize("dim,T,excl,mode,prec,hashed", [(2, 16, 0, 0, 0, False), (2, 24, 1, 1, 1, False),
                                                         (3, 20, 1, 0, 1, True), (3, 32, 0, 2, 0, True),
                                                         (1, 40, 1, 0, 1, False),
                                                         # coarsened bitmaps: the hash keys coarse cells
                                                         (3, 160, 1, 0, 1, True), (3, 200, 1, 1, 0, True)])
def test_filled_cells_count(ug, dim, T, excl, mode, prec, hashed):
    """The device count of occupied (timestep, cell) buckets equals the count from the
    accepted trajectories (the `filled` of braid_cuda.cu:695, 865-879)."""
    from ugb200.cli import filled_cells
    u = ug.Universe(dim=dim, T=T, zgrid=1, excl=excl, seed=3 + T, attempts=20000, group_mode=mode,
                    sub_attempts=20000 if mode == 1 else 0, round_size=2048)
    with ug.Packer([u], precision=prec, force_hash=hashed) as p:
        p.run()
        st = p.stats(0)
        pos = p.positions(0)
    cell = 2.0 / T if excl == 0 else 1.0 / T
    assert st.n > 0 and st.filled == int(filled_cells(pos, cell)[-1])


def test_sub_fill_rate_stop_is_a_prefix(ug):
    """A phase 2 ended by the new-volume stop admits exactly what a budget-limited run to
    the same attempt count admits (same candidate stream, in-order resolution)."""
    kw = dict(dim=2, T=24, zgrid=1, excl=1, seed=4, attempts=20000, group_mode=1, round_size=65536)
    u = ug.Universe(**kw, sub_attempts=60_000_000, sub_fill_rate=5e-4)
    with ug.Packer([u], precision=1) as p:
        p.run()
        st = p.stats(0)
        a, g = p.accepted(0)
    sub = st.attempts - st.phase1_end
    assert 20_000_000 <= sub < 60_000_000
    v = ug.Universe(**kw, sub_attempts=sub)
    with ug.Packer([v], precision=1) as p:
        p.run()
        st2 = p.stats(0)
        b, h = p.accepted(0)
    assert st2.attempts == st.attempts
    assert np.array_equal(a, b) and np.array_equal(g, h)
    assert st2.filled == st.filled


@pytest.mark.parametrize("dim,T,excl,prec,mode", [(2, 32, 0, 0, 0), (2, 32, 1, 1, 0), (3, 24, 1, 1, 0),
                                                   (3, 40, 0, 0, 0), (3, 40, 0, 1, 0), (2, 48, 1, 1, 2),
                                                   (3, 24, 1, 1, 2)])
def test_euclid_exclusion(ug, oracle, dim, T, excl, prec, mode):
    """--euclid-collision (the L2 ball of radius cell, cuda/braid_cuda3d.cu:605-608) on the
    FP64 path and through the tensor-core prefilter's guard band: accepted sets (and
    groups) equal the oracle's."""
    u = ug.Universe(dim=dim, T=T, zgrid=1, excl=excl, seed=21 + T, attempts=30000, euclid=1,
                    group_mode=mode, round_size=2048)
    st, idx = _check(ug, oracle, u, precision=prec)
    cube = ug.Universe(**{**u.__dict__, "euclid": 0})
    with ug.Packer([cube], precision=prec) as p:
        p.run()
        assert p.stats(0).n < st.n  # the ball excludes less than the cube


def test_accepted_all_equals_per_universe(ug):
    """The bulk read-back (one gather, one copy per array) returns what the
    per-universe calls return, and the control-block snapshot is reused between
    reads (no further device-to-host bytes for repeated stats)."""
    us = [ug.Universe(dim=d, T=T, zgrid=1, excl=1, cross1d=int(d == 1), group_mode=g, seed=s,
                      attempts=a, round_size=4096)
          for d, T, g, s, a in [(1, 16, 0, 1, 20000), (2, 24, 2, 2, 30000), (3, 16, 0, 3, 25000),
                                (2, 32, 0, 4, 40000)]]
    with ug.Packer(us, precision=1) as p:
        p.run()
        per = [p.accepted(k) for k in range(len(us))]
        bulk = p.accepted_all()
        for (a, g), (b, h) in zip(per, bulk):
            assert np.array_equal(a, b) and np.array_equal(g, h)
        _, _, d0 = p.counters()
        for k in range(len(us)):
            p.stats(k)
        assert p.counters()[2] == d0


def test_bounded_wait_gives_up_and_context_stays_usable(ug, oracle):
    """A device wait that nothing completes ends after its limit with UG_ETIMEDOUT
    (no trap, no hang), and the context keeps working."""
    import ctypes as C
    import time

    from ugb200 import _lib

    st = C.c_int32(-1)
    t0 = time.perf_counter()
    assert _lib.load().ug_selftest_bounded_wait(50_000_000, C.byref(st)) == 0
    assert st.value == _lib.UG_ETIMEDOUT
    assert time.perf_counter() - t0 >= 0.05
    u = ug.Universe(dim=2, T=16, seed=9, attempts=5000, round_size=1024)
    _check(ug, oracle, u, precision=1)
