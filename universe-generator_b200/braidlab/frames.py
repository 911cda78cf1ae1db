"""Reader of baked .frames files (reference braidlab/frames.py:88-144), the
observer-view remap of a frame's hits on the GPU (frames.py:147-188) and the per-frame
measurements beside it (frames.py:191-223).

The BRF1 layout (cuda/frame_bake.cu:29-38):
  header : b"BRF1", u32 n_paths, u32 n_observers, u32 n_instants, u32 front,
           u32 cheb, f64 speed, f64 z_min, i32 wraps
  observers: u32 type, i32 path_idx, f64 px, f64 py
  per instant: f64 z_obs, f64 chi_max, i32 K, then per observer
           f64 ox, f64 oy, f64 beta_x, f64 beta_y, u64 n_hits, n_hits x
           (u32 src, f32 dx, f32 dy, f32 chi, f32 z_emit)
"""

from __future__ import annotations

import struct
from dataclasses import dataclass
from pathlib import Path

import numpy as np

BETA_CAP = 0.995
FRAME_GRID = 420
FRAME_BISECT = 24
BUDGET_GRID_CAP = 4000
HIT_DTYPE = np.dtype([("src", "<u4"), ("dx", "<f4"), ("dy", "<f4"), ("chi", "<f4"),
                      ("z_emit", "<f4")])
_FRONTS = ("speed", "fit", "budget")


@dataclass(frozen=True)
class ObserverFrame:
    z_obs: float
    chi_max: float
    wraps: int
    ox: float
    oy: float
    beta: np.ndarray
    hits: np.ndarray

    @property
    def redshift(self) -> np.ndarray:
        """Cosmological 1+Z per hit: sin(z_obs) / sin(z_emit)."""
        return np.sin(self.z_obs) / np.sin(self.hits["z_emit"].astype(np.float64))


@dataclass(frozen=True)
class FrameSet:
    n_paths: int
    front: str
    cheb: bool
    speed: float
    z_min: float
    observers: list
    frames: list


def load_frames(path: str | Path) -> FrameSet:
    """Read a .frames file; hits of each frame sorted by (chi, src)."""
    raw = Path(path).read_bytes()
    if raw[:4] != b"BRF1":
        raise ValueError(f"{path}: not a BRF1 frames file")
    n_paths, n_obs, n_inst, front, cheb = struct.unpack_from("<5I", raw, 4)
    speed, z_min = struct.unpack_from("<2d", raw, 24)
    off = 44
    observers = []
    for _ in range(n_obs):
        typ, pidx = struct.unpack_from("<Ii", raw, off)
        px, py = struct.unpack_from("<2d", raw, off + 8)
        observers.append((typ, pidx, px, py))
        off += 24
    frames = []
    for _ in range(n_inst):
        z_obs, chi_max = struct.unpack_from("<2d", raw, off)
        (k,) = struct.unpack_from("<i", raw, off + 16)
        off += 20
        row = []
        for _o in range(n_obs):
            ox, oy, bx, by = struct.unpack_from("<4d", raw, off)
            (nh,) = struct.unpack_from("<Q", raw, off + 32)
            off += 40
            hits = np.frombuffer(raw, dtype=HIT_DTYPE, count=nh, offset=off)
            off += nh * HIT_DTYPE.itemsize
            row.append(ObserverFrame(z_obs, chi_max, k, ox, oy, np.array([bx, by]),
                                     np.sort(hits, order=["chi", "src"])))
        frames.append(row)
    return FrameSet(n_paths, _FRONTS[front], bool(cheb), speed, z_min, observers, frames)


def apparent_positions(frame: ObserverFrame, mode: str = "static", cheb: bool = True):
    """Apparent sky offsets and Doppler log-factor per hit (reference
    braidlab/frames.py:147-188): ``static`` returns the stored offsets (ln_dopp 0);
    ``moving`` boosts each hit's direction into the observer's rest frame by
    ``frame.beta`` (capped at |beta| = 0.995) and puts it back on its own Chebyshev
    shell (``cheb``) or Euclidean one.  Runs on the GPU through libug
    (ug_apparent_positions)."""
    from ugb200.frames import apparent_positions as _apparent

    if mode not in ("static", "moving"):
        raise ValueError(f"mode must be static|moving, got {mode!r}")
    return _apparent(frame.hits, frame.beta, mode, cheb)


def counts_vs_redshift(frame: ObserverFrame, edges: np.ndarray):
    """(histogram, cumulative N(<Z)) of the images binned by cosmological 1+Z
    (frames.py:191-197)."""
    hist, _ = np.histogram(frame.redshift, bins=edges)
    return hist, np.cumsum(hist)


def ghost_multiplicity(frame: ObserverFrame) -> np.ndarray:
    """Images per source worldline: torus wraps and earlier epochs (frames.py:200-202)."""
    return np.bincount(frame.hits["src"])


def load_gids(dump_path: str | Path) -> np.ndarray:
    """Group id per dump row from a subpath dump's trailing gid column
    (frames.py:205-223); a dump without one is an error."""
    import csv

    with open(dump_path) as fh:
        rd = csv.DictReader(fh)
        if rd.fieldnames is None or "gid" not in rd.fieldnames:
            raise ValueError(f"{dump_path}: no gid column (not a subpath dump)")
        return np.array([int(row["gid"]) for row in rd], dtype=np.int64)
