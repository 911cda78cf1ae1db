"""Frame baking of a 2+1 packing on the GPU and the BRF1 writer.

``bake`` runs libug's ug_frame_bake (the frame_bake driver, cuda/frame_bake.cu:398-635)
on dump arrays and returns per-(instant, observer) hit tables and, optionally,
bins x bins uint32 density grids of the hit offsets over [-chi_max, chi_max]^2.
``write_brf1`` writes the reference's .frames layout (cuda/frame_bake.cu:29-38), which
braidlab.frames.load_frames reads.  ``apparent_positions`` is the observer-view remap of a
frame's hits (braidlab/frames.py:147-188) on the GPU.
"""

from __future__ import annotations

import ctypes as C
import struct
from dataclasses import dataclass

import numpy as np

from . import _lib as L

FRONTS = {"speed": 0, "fit": 1, "budget": 2}
HIT_DTYPE = np.dtype([("src", "<u4"), ("dx", "<f4"), ("dy", "<f4"), ("chi", "<f4"),
                      ("z_emit", "<f4")])


class _Cfg(C.Structure):
    _fields_ = [("front", C.c_int32), ("cheb", C.c_int32), ("n_frames", C.c_int32),
                ("wraps", C.c_int32), ("from_pi", C.c_double), ("to_pi", C.c_double),
                ("zmin_pi", C.c_double), ("speed", C.c_double), ("n_obs", C.c_int32),
                ("density_bins", C.c_int32), ("obs_type", C.c_void_p), ("obs_path", C.c_void_p),
                ("obs_xy", C.c_void_p)]


class _Out(C.Structure):
    _fields_ = [("hits", C.c_void_p), ("hit_cap", C.c_int64), ("hit_count", C.c_void_p),
                ("frame_meta", C.c_void_p), ("obs_meta", C.c_void_p), ("density", C.c_void_p),
                ("hits_total", C.c_int64)]


@dataclass
class Baked:
    front: str
    cheb: bool
    speed: float
    z_min: float
    wraps: int
    observers: list          # (type, path_idx, px, py)
    frame_meta: np.ndarray   # [frames][3] z_obs, chi_max, K
    obs_meta: np.ndarray     # [frames][obs][4] ox, oy, beta_x, beta_y
    hits: list | None        # [frames][obs] -> HIT_DTYPE arrays sorted by (chi, src); None: not kept
    density: np.ndarray | None  # [frames][obs][bins][bins] uint32
    n_paths: int
    counts: np.ndarray | None = None  # [frames][obs] hits per (frame, observer)


def _bake(call, n, *, observers, from_pi, to_pi, frames, zmin_pi, front, metric, speed, wraps,
          density_bins, hit_cap, hits) -> Baked:
    ot = np.array([0 if o[0] == "path" else 1 for o in observers], np.int32)
    op = np.array([o[1] if o[0] == "path" else -1 for o in observers], np.int32)
    oxy = np.array([[0.0, 0.0] if o[0] == "path" else [o[1], o[2]] for o in observers], np.float64)
    cheb = 1 if (front == "budget" or metric == "square") else 0
    cfg = _Cfg(FRONTS[front], cheb, frames, wraps, from_pi, to_pi, zmin_pi, speed, len(observers),
               density_bins, ot.ctypes.data, op.ctypes.data, oxy.ctypes.data)
    hbuf = np.empty(hit_cap, HIT_DTYPE) if hits else None
    counts = np.zeros((frames, len(observers)), np.int64)
    fmeta = np.zeros((frames, 3))
    ometa = np.zeros((frames, len(observers), 4))
    den = (np.empty((frames, len(observers), density_bins, density_bins), np.uint32)
           if density_bins else None)
    out = _Out(hbuf.ctypes.data if hbuf is not None else None, hit_cap if hits else 0,
               counts.ctypes.data, fmeta.ctypes.data, ometa.ctypes.data,
               den.ctypes.data if den is not None else None, 0)
    L.check(call(C.byref(cfg), C.byref(out)))
    per = None
    if hits:
        per, k = [], 0
        for fi in range(frames):
            row = []
            for o in range(len(observers)):
                c = int(counts[fi, o])
                row.append(hbuf[k:k + c].copy())
                k += c
            per.append(row)
    obs = [(int(ot[i]), int(op[i]), float(oxy[i, 0]), float(oxy[i, 1])) for i in range(len(observers))]
    return Baked(front, bool(cheb), speed, max(2e-3, zmin_pi * np.pi), wraps, obs, fmeta, ometa, per,
                 den, n, counts)


def bake(a2, a, b, f, *, observers, from_pi=0.25, to_pi=0.75, frames=1, zmin_pi=0.02,
         front="fit", metric="square", speed=0.33, wraps=-1, density_bins=0,
         hit_cap=1 << 22, hits=True) -> Baked:
    """Frames of dump arrays a2 [n][2], a/b/f [n][2][nw] (host memory).
    observers: list of ("path", idx) or ("point", x, y).  hits=False keeps only the
    hit counts and densities (no per-frame wait for the host)."""
    lib = L.load()
    a2 = np.ascontiguousarray(a2, np.float64)
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    f = np.ascontiguousarray(f, np.float64)
    n, _, nw = a.shape
    return _bake(lambda cfg, out: lib.ug_frame_bake(cfg, n, nw, a2.ctypes.data, a.ctypes.data,
                                                    b.ctypes.data, f.ctypes.data, out), n,
                 observers=observers, from_pi=from_pi, to_pi=to_pi, frames=frames, zmin_pi=zmin_pi,
                 front=front, metric=metric, speed=speed, wraps=wraps, density_bins=density_bins,
                 hit_cap=hit_cap, hits=hits)


def bake_packed(packer, u=0, *, observers, from_pi=0.25, to_pi=0.75, frames=1, zmin_pi=0.02,
                front="fit", metric="square", speed=0.33, wraps=-1, density_bins=0,
                hit_cap=1 << 22, hits=True) -> Baked:
    """Frames of universe u of a Packer (2+1) baked from its device-resident paths: the
    dump -> frame_bake pipeline without the CSV.  Path indices are admission order."""
    lib = L.load()
    n = packer.stats(u).n
    return _bake(lambda cfg, out: lib.ug_batch_frames(packer._h, u, cfg, out), n,
                 observers=observers, from_pi=from_pi, to_pi=to_pi, frames=frames, zmin_pi=zmin_pi,
                 front=front, metric=metric, speed=speed, wraps=wraps, density_bins=density_bins,
                 hit_cap=hit_cap, hits=hits)


def write_brf1(path, bk: Baked) -> None:
    """The reference's .frames file (little-endian), cuda/frame_bake.cu:29-38, 485-623."""
    with open(path, "wb") as fh:
        fh.write(b"BRF1")
        fh.write(struct.pack("<3I", bk.n_paths, len(bk.observers), len(bk.hits)))
        fh.write(struct.pack("<2I", FRONTS[bk.front], int(bk.cheb)))
        fh.write(struct.pack("<d", bk.speed))
        fh.write(struct.pack("<d", bk.z_min))
        fh.write(struct.pack("<i", bk.wraps))
        for t, p, x, y in bk.observers:
            fh.write(struct.pack("<Ii", t, p if t == 0 else -1))
            fh.write(struct.pack("<2d", x, y))
        for fi, row in enumerate(bk.hits):
            z, chi, K = bk.frame_meta[fi]
            fh.write(struct.pack("<2d", z, chi))
            fh.write(struct.pack("<i", int(K)))
            for o, h in enumerate(row):
                fh.write(struct.pack("<4d", *bk.obs_meta[fi, o]))
                fh.write(struct.pack("<Q", len(h)))
                fh.write(h.astype(HIT_DTYPE).tobytes())


VIEW_MODES = {"static": 0, "moving": 1}


def apparent_positions(hits: np.ndarray, beta, mode: str = "static", cheb: bool = True):
    """(ax, ay, ln_dopp) of HIT_DTYPE hits seen by an observer of boost ``beta``
    (braidlab/frames.py:147-188) through ug_apparent_positions: ``static`` keeps the
    stored offsets; ``moving`` aberrates each hit's direction into the observer's rest
    frame (|beta| capped at 0.995) with the Doppler log-factor, on the Chebyshev shell
    of its chi when ``cheb``."""
    if mode not in VIEW_MODES:
        raise ValueError(f"mode must be static|moving, got {mode!r}")
    h = np.ascontiguousarray(hits, dtype=HIT_DTYPE)
    n = len(h)
    out = np.empty((3, n), np.float64)
    bx, by = (float(v) for v in np.asarray(beta, np.float64).reshape(2))
    lib = L.load()
    L.check(lib.ug_apparent_positions(h.ctypes.data if n else None, n, bx, by, VIEW_MODES[mode],
                                      int(bool(cheb)), out[0].ctypes.data, out[1].ctypes.data,
                                      out[2].ctypes.data))
    return out[0], out[1], out[2]
