"""The allocation-free parameter dump (ug_batch_params_noalloc) against the
allocating one (ug_batch_params), through the C ABI.

Collected last (file name), so a run that stops at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dump(lib, fn, h, u, n, dim, nw):
    a2 = np.zeros((n, dim))
    a = np.zeros((n, dim, nw))
    f = np.zeros((n, dim, nw))
    b = np.zeros((n, dim, nw), np.int32)
    rc = getattr(lib, fn)(h, u, a2.ctypes.data, a.ctypes.data, b.ctypes.data, f.ctypes.data, n)
    return rc, a2, a, b, f


def test_noalloc_params_match_allocating_dump(ug):
    from ugb200 import _lib

    us = [ug.Universe(dim=2, T=32, zgrid=1, excl=1, seed=7, attempts=40000, round_size=4096),
          ug.Universe(dim=3, T=16, rng=1, seed=3, attempts=20000, round_size=4096)]
    with ug.Packer(us) as p:
        p.run()
        lib = _lib.load()
        for k, u in enumerate(us):
            n = p.stats(k).n
            assert n > 0
            ref = _dump(lib, "ug_batch_params", p._h, k, n, u.dim, u.nw)
            assert ref[0] == 0
            for _ in range(2):  # two calls in a row share the fixed stage
                got = _dump(lib, "ug_batch_params_noalloc", p._h, k, n, u.dim, u.nw)
                assert got[0] == 0, _lib.last_error()
                for x, y in zip(ref[1:], got[1:]):
                    assert np.array_equal(x, y)  # same kernel, same inputs: bit-identical


def test_noalloc_rejects_dumps_beyond_the_stage(ug):
    from ugb200 import _lib

    # 3 axes x 255 terms: ~15 KB per path, so a few thousand paths exceed 16 MiB
    u = ug.Universe(dim=3, T=256, zgrid=1, excl=1, seed=1, attempts=3000, round_size=1024)
    with ug.Packer([u]) as p:
        p.run()
        n = p.stats(0).n
        assert n * 3 * (8 + 20 * 255) > (16 << 20)
        rc = _dump(_lib.load(), "ug_batch_params_noalloc", p._h, 0, n, 3, 255)[0]
        assert rc == _lib.UG_ECAP
        assert "16777216" in _lib.last_error()
