"""frame_bake on the GPU against the reference's own Python baker (golden hits),
plus the reference test's properties, the BRF1 round trip and the density scatter."""

import io
import json
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "frames_reference.json")
TOL = 2e-5  # float32 hit records; positions agree to ~1e-13 in FP64


def _arrays(text):
    import tempfile

    from ugb200.io import load_dump
    with tempfile.NamedTemporaryFile("w", suffix=".csv", delete=False) as fh:
        fh.write(text)
        p = fh.name
    dim, a2, a, b, f, _ = load_dump(p)
    os.remove(p)
    return a2, a, b, f


def _bake_case(ug, c, dumps, **kw):
    from ugb200.frames import bake
    a2, a, b, f = _arrays(dumps[c["dump"]])
    obs = [tuple(c["obs"])]
    return bake(a2, a, b, f, observers=obs, from_pi=c["z_obs_pi"], to_pi=c["z_obs_pi"], frames=1,
                zmin_pi=c["z_min_pi"], front=c["front"], metric="square" if c["cheb"] else "circle",
                speed=c["speed"], wraps=-1 if c["wraps"] is None else c["wraps"], **kw)


def test_hits_match_reference_baker(ug):
    gold = json.load(open(GOLD))
    for k, c in enumerate(gold["cases"]):
        bk = _bake_case(ug, c, gold["dumps"])
        got = bk.hits[0][0]
        ref = np.array(c["hits"], dtype=float).reshape(-1, 5)
        assert len(got) == len(ref), (k, len(got), len(ref))
        if not len(ref):
            continue
        # pair hits by (src, chi, dx, dy): images of one source can share chi
        key = lambda m: np.lexsort((np.round(m[:, 2], 4), np.round(m[:, 1], 4),  # noqa: E731
                                    np.round(m[:, 3], 5), m[:, 0]))
        ref = ref[key(ref)]
        gg = np.stack([got["src"].astype(float), got["dx"], got["dy"], got["chi"], got["z_emit"]], 1)
        gg = gg[key(gg)]
        assert np.array_equal(gg[:, 0], ref[:, 0]), k
        np.testing.assert_allclose(gg[:, 1:], ref[:, 1:], atol=TOL, rtol=0)


def test_reference_properties_on_packed_dump(ug):
    """Hits sit on the front, emit times lie in the rewind window (tests/test_frames.py:34-45)."""
    gold = json.load(open(GOLD))
    a2, a, b, f = _arrays(gold["dumps"]["packed"])
    from ugb200.frames import bake
    for front in ("fit", "budget", "speed"):
        bk = bake(a2, a, b, f, observers=[("path", 0), ("point", 0.2, -0.1)], from_pi=0.3,
                  to_pi=0.7, frames=3, zmin_pi=0.02, front=front)
        for fi in range(3):
            z_obs = bk.frame_meta[fi, 0]
            for o in range(2):
                h = bk.hits[fi][o]
                assert len(h) > 0
                assert np.all(h["src"] < len(a2))
                assert np.all(h["z_emit"] <= z_obs + 1e-5) and np.all(h["z_emit"] >= 0.02 * math.pi - 1e-5)
                r = np.maximum(np.abs(h["dx"]), np.abs(h["dy"]))
                np.testing.assert_allclose(r, h["chi"], atol=1e-5)


def test_brf1_round_trip_and_density(ug, tmp_path):
    from braidlab.frames import load_frames
    from ugb200.frames import bake, write_brf1
    gold = json.load(open(GOLD))
    a2, a, b, f = _arrays(gold["dumps"]["packed"])
    bins = 64
    bk = bake(a2, a, b, f, observers=[("path", 2)], from_pi=0.3, to_pi=0.7, frames=4,
              zmin_pi=0.02, front="fit", density_bins=bins)
    p = tmp_path / "x.frames"
    write_brf1(p, bk)
    fs = load_frames(p)
    assert fs.n_paths == len(a2) and fs.front == "fit" and len(fs.frames) == 4
    for fi in range(4):
        fr = fs.frames[fi][0]
        assert np.array_equal(fr.hits, np.sort(bk.hits[fi][0], order=["chi", "src"]))
        chi_max = bk.frame_meta[fi, 1]
        h = bk.hits[fi][0]
        cx = np.floor((h["dx"].astype(np.float32) + np.float32(chi_max)) * np.float32(bins / (2 * chi_max)))
        cy = np.floor((h["dy"].astype(np.float32) + np.float32(chi_max)) * np.float32(bins / (2 * chi_max)))
        # closed square: an offset rounded a hair past an edge counts in the edge bin
        cx = np.clip(cx, 0, bins - 1).astype(int)
        cy = np.clip(cy, 0, bins - 1).astype(int)
        ref = np.zeros((bins, bins), np.uint32)
        np.add.at(ref, (cy, cx), 1)
        assert np.array_equal(bk.density[fi, 0], ref)
        assert int(bk.density[fi, 0].sum()) == len(h)


def test_device_pipeline_equals_host_arrays(ug):
    """Frames baked from the packer's device-resident paths equal frames baked from the
    same paths' dump arrays; the density-only mode returns the same counts and grids."""
    from ugb200.frames import bake, bake_packed
    u = ug.Universe(dim=2, T=32, zgrid=1, excl=1, seed=9, attempts=30000, round_size=4096)
    kw = dict(observers=[("path", 3), ("point", 0.1, -0.2)], from_pi=0.3, to_pi=0.7, frames=5,
              zmin_pi=0.02, front="fit", density_bins=128)
    with ug.Packer([u], precision=ug.PREC_MIXED) as p:
        p.run()
        par = p.params(0)
        dev = bake_packed(p, 0, **kw)
        dev_d = bake_packed(p, 0, hits=False, **kw)
    host = bake(par["a2"], par["a"], par["b"], par["f"], **kw)
    host_d = bake(par["a2"], par["a"], par["b"], par["f"], hits=False, **kw)
    assert dev.n_paths == host.n_paths == len(par["a2"])
    np.testing.assert_array_equal(dev.frame_meta, host.frame_meta)
    np.testing.assert_array_equal(dev.obs_meta, host.obs_meta)
    order = ["chi", "src", "dx", "dy", "z_emit"]  # (chi, src) ties come in device order
    for fi in range(5):
        for o in range(2):
            x, y = np.sort(dev.hits[fi][o], order=order), np.sort(host.hits[fi][o], order=order)
            assert len(x) == len(y) == dev_d.counts[fi, o] == host_d.counts[fi, o]
            diff = np.nonzero(x != y)[0]
            assert diff.size == 0, (fi, o, x[diff[:3]], y[diff[:3]])
    assert dev.counts.sum() > 0
    for d in (dev_d, host, host_d):
        assert np.array_equal(d.density, dev.density)
    assert int(dev.density.sum()) == int(dev.counts.sum())
