"""Mixed-precision (tensor-core split-BF16) prefilter: achieved position error
against FP64 and exact accepted-set parity with the FP64 path and the oracle."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _model(O, u):
    return O.Model(dim=u.dim, T=u.T, terms=u.terms, rng=u.rng, zgrid=u.zgrid, excl=u.excl,
                   cross1d=u.cross1d, pin=u.pin_sin1, seed=u.seed, euclid=u.euclid)


@pytest.mark.parametrize("dim,T,zg,ex,cx", [(2, 16, 0, 0, 0), (2, 64, 1, 1, 0), (3, 128, 1, 1, 0),
                                            (3, 200, 1, 1, 0), (2, 23, 0, 1, 0), (1, 256, 1, 0, 0),
                                            (1, 40, 1, 1, 1)])
def test_mixed_position_error_within_guard(ug, dim, T, zg, ex, cx):
    u = ug.Universe(dim=dim, T=T, zgrid=zg, excl=ex, cross1d=cx, seed=3, attempts=1000, round_size=1024)
    with ug.Packer([u], precision=ug.PREC_MIXED) as p:
        err, margin, ratio = p.mixed_error(0, 0, 2048)
    print(f"dim={dim} T={T}: max |X_mixed - X_fp64| = {err:.3e}, widest guard {margin:.3e}, "
          f"max error / own guard {ratio:.3e}")
    assert err < margin / 2
    # the guard band of every (candidate, timestep) is twice its rigorous error bound
    assert ratio < 0.5


@pytest.mark.parametrize("dim,T,zg,ex,att", [(2, 16, 0, 0, 30000), (2, 32, 1, 1, 60000),
                                             (3, 24, 1, 1, 40000), (2, 64, 1, 1, 100000),
                                             (3, 200, 1, 1, 8000), (2, 23, 0, 1, 30000),
                                             (3, 240, 1, 1, 6000), (2, 250, 1, 1, 40000)])
def test_mixed_accepted_set_equals_oracle_and_fp64(ug, oracle, dim, T, zg, ex, att):
    u = ug.Universe(dim=dim, T=T, zgrid=zg, excl=ex, seed=11 + T, attempts=att, round_size=4096)
    ref = oracle.pack(_model(oracle, u), att)
    with ug.Packer([u], precision=ug.PREC_MIXED) as p:
        p.run()
        a, _ = p.accepted(0)
        st = p.stats(0)
    with ug.Packer([u], precision=ug.PREC_FP64) as p:
        p.run()
        b, _ = p.accepted(0)
    assert np.array_equal(a, b)
    assert np.array_equal(a, ref.acc_idx)
    print(f"dim={dim} T={T}: N={len(a)} gray={st.gray} evals={st.evals} fp64 evals={st.evals_fp64}")


def test_mixed_batch_with_fp64_only_universes(ug, oracle):
    """Knot-stream and 1+1D crossing universes take the FP64 path inside a mixed batch."""
    us = [ug.Universe(dim=2, T=16, seed=1, attempts=20000, round_size=2048),
          ug.Universe(dim=2, T=16, rng=1, seed=2, attempts=20000, round_size=2048),
          ug.Universe(dim=1, T=16, zgrid=1, excl=1, cross1d=1, seed=3, attempts=20000,
                      round_size=2048),
          ug.Universe(dim=3, T=32, zgrid=1, excl=1, seed=4, attempts=20000, round_size=2048)]
    with ug.Packer(us, precision=ug.PREC_MIXED) as p:
        p.run()
        for k, u in enumerate(us):
            idx, _ = p.accepted(k)
            ref = oracle.pack(_model(oracle, u), u.attempts)
            assert np.array_equal(idx, ref.acc_idx), k


@pytest.mark.parametrize("T,seed", [(16, 3), (40, 8), (101, 2)])
def test_mixed_1d_crossing_rule(ug, oracle, T, seed):
    """1+1D with the crossing rule through the tensor-core path (guard-banded FP32
    contact and sign-change test, FP64 retest of the undecided)."""
    u = ug.Universe(dim=1, T=T, zgrid=1, excl=1, cross1d=1, seed=seed, attempts=30000, round_size=4096)
    ref = oracle.pack(_model(oracle, u), u.attempts)
    with ug.Packer([u], precision=ug.PREC_MIXED) as p:
        p.run()
        a, _ = p.accepted(0)
        st = p.stats(0)
    assert np.array_equal(a, ref.acc_idx)
    assert st.gray < u.attempts // 10  # most candidates decided in FP32
