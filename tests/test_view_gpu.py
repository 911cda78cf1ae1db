"""Observer-view remap on the GPU (ug_apparent_positions) against the reference's own
outputs (golden) and the oracle (braidlab/frames.py:147-188), through the C ABI."""

import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "view_reference.json")
# FP64 with every product and sum rounded as the reference rounds it; hypot and log
# are CUDA's (within 1-2 ulp of the host libm).  The boost amplifies those ulps by up
# to ~gamma^2 (1 + beta) ~ 200 at the 0.995 cap, so offsets agree to 1e-12 of the
# hit's shell radius chi (2.2e-13 absolute seen at chi <= 4 over 2^20 hits), and the
# Doppler log-factor to 1e-13.
RTOL, ATOL = 1e-13, 1e-13
SHELL_TOL = 1e-12


def _close_offsets(got, want, chi):
    chi = np.asarray(chi, np.float32).astype(np.float64)
    err = np.abs(np.asarray(got) - np.asarray(want))
    bad = err > RTOL * np.abs(want) + SHELL_TOL * chi
    assert not bad.any(), f"{bad.sum()} offsets off by up to {err[bad].max():.3g}"


def _hits(dx, dy, chi):
    from ugb200.frames import HIT_DTYPE

    h = np.zeros(len(dx), HIT_DTYPE)
    h["dx"], h["dy"], h["chi"] = dx, dy, chi
    h["src"] = np.arange(len(h))
    return h


def test_remap_matches_reference_golden(ug):
    from ugb200.frames import apparent_positions

    for c in json.load(open(GOLD)):
        ax, ay, ld = apparent_positions(_hits(c["dx"], c["dy"], c["chi"]), c["beta"], c["mode"], c["cheb"])
        _close_offsets(ax, c["ax"], c["chi"])
        _close_offsets(ay, c["ay"], c["chi"])
        np.testing.assert_allclose(ld, c["ln_dopp"], rtol=RTOL, atol=ATOL)
        if c["mode"] == "static" or np.hypot(*c["beta"]) <= 1e-6:  # copies: exact
            assert np.array_equal(ax, c["ax"]) and np.array_equal(ld, c["ln_dopp"])


@pytest.mark.parametrize("beta", [(0.6, -0.3), (3.0, 4.0), (0.0, 1e-3)])
@pytest.mark.parametrize("cheb", [True, False])
def test_remap_matches_oracle_at_scale(ug, oracle, beta, cheb):
    from ugb200.frames import apparent_positions

    rng = np.random.default_rng(11)
    n = 1 << 20
    chi = rng.uniform(1e-3, 4.0, n).astype(np.float32)
    ang = rng.uniform(-np.pi, np.pi, n)
    dx = (chi * np.cos(ang)).astype(np.float32)
    dy = (chi * np.sin(ang)).astype(np.float32)
    dx[::997] = 0.0
    dy[::997] = 0.0
    ax, ay, ld = apparent_positions(_hits(dx, dy, chi), beta, "moving", cheb)
    ox, oy, ol = oracle.apparent_positions(dx, dy, chi, beta, "moving", cheb)
    _close_offsets(ax, ox, chi)
    _close_offsets(ay, oy, chi)
    np.testing.assert_allclose(ld, ol, rtol=RTOL, atol=ATOL)
    # size-independent properties: images stay on their own shell, centre hits stay put
    r = np.maximum(np.abs(ax), np.abs(ay)) if cheb else np.hypot(ax, ay)
    moved = (dx != 0) | (dy != 0)
    np.testing.assert_allclose(r[moved], chi[moved].astype(np.float64), rtol=1e-12)
    assert np.all(ax[~moved] == 0) and np.all(ld[~moved] == 0)


def test_async_entry_on_device_buffers(ug, oracle):
    import ctypes

    import torch
    from ugb200 import _lib

    rng = np.random.default_rng(4)
    n = 4096
    chi = rng.uniform(0.1, 2.0, n).astype(np.float32)
    dx = (chi * rng.uniform(-1, 1, n)).astype(np.float32)
    dy = (chi * rng.uniform(-1, 1, n)).astype(np.float32)
    h = _hits(dx, dy, chi)
    dh = torch.from_numpy(h.view(np.uint8).copy()).cuda()
    out = torch.empty((3, n), dtype=torch.float64, device="cuda")
    st = torch.cuda.Stream()
    lib = _lib.load()
    rc = lib.ug_apparent_positions_async(dh.data_ptr(), n, -0.4, 0.45, 1, 1, out[0].data_ptr(),
                                         out[1].data_ptr(), out[2].data_ptr(), ctypes.c_void_p(st.cuda_stream))
    assert rc == 0, _lib.last_error()
    st.synchronize()
    got = out.cpu().numpy()
    want = oracle.apparent_positions(dx, dy, chi, (-0.4, 0.45), "moving", True)
    _close_offsets(got[0], want[0], chi)
    _close_offsets(got[1], want[1], chi)
    np.testing.assert_allclose(got[2], want[2], rtol=RTOL, atol=ATOL)


def test_mirror_remap_of_a_baked_frame(ug, oracle, tmp_path):
    """braidlab.frames.apparent_positions on a frame read back from a BRF1 file the
    packer's device bake wrote, against the oracle on the same hits."""
    from braidlab.frames import apparent_positions, load_frames
    from ugb200.frames import bake_packed, write_brf1

    u = ug.Universe(dim=2, T=32, zgrid=1, excl=1, seed=5, attempts=30000, round_size=4096)
    with ug.Packer([u], precision=ug.PREC_MIXED) as p:
        p.run()
        bk = bake_packed(p, 0, observers=[("path", 3), ("point", 0.1, -0.2)], from_pi=0.3, to_pi=0.7,
                         frames=2, front="fit")
    path = tmp_path / "u.frames"
    write_brf1(path, bk)
    fs = load_frames(path)
    seen = 0
    for row in fs.frames:
        for fr in row:
            for mode in ("static", "moving"):
                ax, ay, ld = apparent_positions(fr, mode, fs.cheb)
                ox, oy, ol = oracle.apparent_positions(fr.hits["dx"], fr.hits["dy"], fr.hits["chi"], fr.beta,
                                                       mode, fs.cheb)
                _close_offsets(ax, ox, fr.hits["chi"])
                _close_offsets(ay, oy, fr.hits["chi"])
                np.testing.assert_allclose(ld, ol, rtol=RTOL, atol=ATOL)
            seen += len(fr.hits)
    assert seen > 0 and np.hypot(*fs.frames[0][0].beta) > 1e-6  # the path observer moves
