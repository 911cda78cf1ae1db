"""CPU oracle for the RSA worldline packer -- TEST INFRASTRUCTURE ONLY.

ctypes bindings to ``libug_oracle.so`` (a plain-C restatement of the
reference's packing path, see ``ug_oracle.c`` for the file:line map) and to
the reference-derived checkers under ``_ref/``.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline legs use this
package; the packer never imports it.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libug_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

RNG_PHILOX, RNG_KNOT = 0, 1
ZGRID_REF, ZGRID_MID = 0, 1
EXCL_REF, EXCL_OPEN = 0, 1
GROUP_NONE, GROUP_SUBPATH, GROUP_UNIQUE = 0, 1, 2


class _Model(C.Structure):
    _fields_ = [
        ("dim", C.c_int32),
        ("T", C.c_int32),
        ("nw", C.c_int32),
        ("rng", C.c_int32),
        ("zgrid", C.c_int32),
        ("excl", C.c_int32),
        ("cross1d", C.c_int32),
        ("pin", C.c_int32),
        ("euclid", C.c_int32),
        ("seed", C.c_uint64),
    ]


class _Run(C.Structure):
    _fields_ = [
        ("attempts", C.c_int64),
        ("max_n", C.c_int64),
        ("group_mode", C.c_int32),
        ("nthreads", C.c_int32),
        ("sub_attempts", C.c_int64),
        ("round", C.c_int64),
        ("accept_rate", C.c_double),
        ("sub_accept_rate", C.c_double),
        ("sub_fill_rate", C.c_double),
    ]


class _Result(C.Structure):
    _fields_ = [
        ("cap", C.c_int64),
        ("acc_idx", C.POINTER(C.c_int64)),
        ("gid", C.POINTER(C.c_int32)),
        ("n_acc", C.c_int64),
        ("n_unique", C.c_int64),
        ("n_sub", C.c_int64),
        ("attempts", C.c_int64),
        ("phase1_end", C.c_int64),
    ]


_lib = None

# Where the checkers read the reference's sources: UG_REFERENCE, else the default of
# the build recipe in this folder's Makefile.  Only this module, the Makefile and the
# test infrastructure that imports REFERENCE_DIR (parity tests, fixture generators)
# read the reference; nothing in the package does.
REFERENCE_DIR = os.environ.get("UG_REFERENCE", "/root/reference")


def build() -> None:
    """Compile libug_oracle.so (and the reference checkers when the tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE, "libug_oracle.so"], check=True)
    if os.path.isdir(REFERENCE_DIR + "/cuda"):
        subprocess.run(["make", "-s", "-C", HERE, "ref", "UG_REFERENCE=" + REFERENCE_DIR], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.ora_philox4x32_10.argtypes = [C.POINTER(C.c_uint32)] * 3
        L.ora_xoshiro_stream.argtypes = [C.c_uint64, C.c_int32, C.POINTER(C.c_uint64)]
        L.ora_candidate.argtypes = [C.POINTER(_Model), C.c_uint64] + [C.c_void_p] * 6
        L.ora_candidate.restype = C.c_int
        L.ora_positions.argtypes = [C.POINTER(_Model), C.c_uint64, C.c_void_p]
        L.ora_positions.restype = C.c_int
        L.ora_tables.argtypes = [C.POINTER(_Model)] + [C.c_void_p] * 4
        L.ora_tables.restype = C.c_int
        L.ora_pack.argtypes = [C.POINTER(_Model), C.POINTER(_Run), C.POINTER(_Result)]
        L.ora_pack.restype = C.c_int
        _lib = L
    return _lib


@dataclass
class Model:
    dim: int = 2
    T: int = 16
    terms: int = 0  # 0 = full band (nw = T-1)
    rng: int = RNG_PHILOX
    zgrid: int = ZGRID_REF
    excl: int = EXCL_REF
    cross1d: int = 0
    pin: int = 0
    seed: int = 0
    euclid: int = 0  # --euclid-collision: L2 ball instead of the Chebyshev cube

    @property
    def nw(self) -> int:
        return (self.terms or self.T) - 1

    def _c(self) -> _Model:
        return _Model(self.dim, self.T, self.nw, self.rng, self.zgrid, self.excl,
                      self.cross1d, self.pin, self.euclid, self.seed & (2**64 - 1))


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def philox(ctr, key) -> np.ndarray:
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().ora_philox4x32_10(c, k, o)
    return np.array(list(o), dtype=np.uint32)


def xoshiro_stream(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, dtype=np.uint64)
    lib().ora_xoshiro_stream(seed, n, out.ctypes.data_as(C.POINTER(C.c_uint64)))
    return out


def candidate(m: Model, idx: int) -> dict:
    d, nw, T = m.dim, m.nw, m.T
    b = np.zeros((d, nw), np.int32)
    a = np.zeros((d, nw))
    f = np.zeros((d, nw))
    a2 = np.zeros(d)
    al = np.zeros((d, T + 1))
    be = np.zeros((d, T + 1))
    mc = m._c()
    rc = lib().ora_candidate(C.byref(mc), idx, _p(b), _p(a), _p(f), _p(a2), _p(al), _p(be))
    if rc:
        raise ValueError("bad model")
    return {"b": b, "a": a, "f": f, "a2": a2, "alpha": al, "beta": be}


def positions(m: Model, idx: int) -> np.ndarray:
    out = np.zeros((m.dim, m.T))
    mc = m._c()
    if lib().ora_positions(C.byref(mc), idx, _p(out)):
        raise ValueError("bad model")
    return out


def tables(m: Model):
    T = m.T
    z = np.zeros(T)
    inv = np.zeros(T)
    S = np.zeros((T + 1, T))
    Cc = np.zeros((T + 1, T))
    mc = m._c()
    if lib().ora_tables(C.byref(mc), _p(z), _p(inv), _p(S), _p(Cc)):
        raise ValueError("bad model")
    return z, inv, S, Cc


@dataclass
class PackResult:
    acc_idx: np.ndarray
    gid: np.ndarray
    n_unique: int
    n_sub: int
    attempts: int
    phase1_end: int


def pack(m: Model, attempts: int, *, max_n: int = 0, group_mode: int = GROUP_NONE,
         sub_attempts: int = 0, nthreads: int = 1, round_size: int = 65536,
         accept_rate: float = 0.0, sub_accept_rate: float = 0.0, sub_fill_rate: float = 0.0,
         cap: int | None = None) -> PackResult:
    """Sequential RSA over the candidate stream (nthreads > 1: threaded batch
    prefilter + in-order decisions, same result).  The windowed stops use
    buckets of win_target / 32 candidates aligned at the phase start."""
    cap = cap or max(1024, attempts + (sub_attempts or (attempts if group_mode == GROUP_SUBPATH else 0)))
    acc = np.zeros(cap, np.int64)
    gid = np.zeros(cap, np.int32)
    res = _Result(cap, acc.ctypes.data_as(C.POINTER(C.c_int64)),
                  gid.ctypes.data_as(C.POINTER(C.c_int32)), 0, 0, 0, 0, 0)
    run = _Run(attempts, max_n, group_mode, nthreads, sub_attempts, round_size,
               accept_rate, sub_accept_rate, sub_fill_rate)
    mc = m._c()
    rc = lib().ora_pack(C.byref(mc), C.byref(run), C.byref(res))
    if rc:
        raise RuntimeError(f"ora_pack failed ({rc})")
    n = res.n_acc
    return PackResult(acc[:n].copy(), gid[:n].copy(), res.n_unique, res.n_sub,
                      res.attempts, res.phase1_end)


def knot_host(args: list[str]) -> subprocess.CompletedProcess:
    """Run the reference-derived CPU checker (oracle/_ref/knot_host)."""
    exe = os.path.join(REF_DIR, "knot_host")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    return subprocess.run([exe] + args, capture_output=True, text=True, check=True)


def parse_knot_dump(text: str, dim: int, nw: int):
    """Rows of a braid_knot --dump file (species, attempt, per axis a2 + nw x (b,a,f))."""
    rows = []
    for line in text.splitlines():
        if not line or line.startswith("#"):
            continue
        v = line.split(",")
        species, attempt = int(v[0]), int(v[1])
        k = 2
        b = np.zeros((dim, nw), np.int32)
        a = np.zeros((dim, nw))
        f = np.zeros((dim, nw))
        a2 = np.zeros(dim)
        for ax in range(dim):
            a2[ax] = float(v[k]); k += 1
            for j in range(nw):
                b[ax, j] = int(v[k]); a[ax, j] = float(v[k + 1]); f[ax, j] = float(v[k + 2])
                k += 3
        rows.append({"species": species, "idx": attempt - 1, "b": b, "a": a, "f": f, "a2": a2})
    return rows


# ---------------------------------------------------------------------------
# Observer-view remap of a frame's hits (numpy restatement of the reference's
# braidlab/frames.py:147-188, apparent_positions).  FP64 throughout, the
# reference's operations in its order.
# ---------------------------------------------------------------------------

BETA_CAP = 0.995  # braidlab/frames.py:37


def apparent_positions(dx, dy, chi, beta, mode: str = "static", cheb: bool = True):
    """(ax, ay, ln_dopp) for float32 hit offsets dx, dy and front radii chi seen by
    an observer of boost beta: frames.py:159-162 (static), 163-174 (boost set-up:
    cap, static below 1e-6, gamma, unit vector), 175-188 (per-hit aberration,
    Doppler factor, Chebyshev or Euclidean shell)."""
    dx = np.asarray(dx, np.float32).astype(np.float64)
    dy = np.asarray(dy, np.float32).astype(np.float64)
    if mode == "static":
        return dx, dy, np.zeros(len(dx))
    if mode != "moving":
        raise ValueError(f"mode must be static|moving, got {mode!r}")
    b = np.array(beta, np.float64).reshape(2)
    bm = float(np.hypot(b[0], b[1]))
    if bm > BETA_CAP:
        b = b * (BETA_CAP / bm)
        bm = BETA_CAP
    if bm <= 1e-6:
        return dx, dy, np.zeros(len(dx))
    g = 1.0 / np.sqrt(1.0 - bm ** 2)
    ux, uy = b[0] / bm, b[1] / bm
    r = np.hypot(dx, dy)
    ok = r > 0
    nx = np.where(ok, dx / np.where(ok, r, 1.0), 0.0)
    ny = np.where(ok, dy / np.where(ok, r, 1.0), 0.0)
    bn = b[0] * nx + b[1] * ny
    un = ux * nx + uy * ny
    dfac = g * (1.0 + bn)
    px = (nx + g * b[0] + (g - 1.0) * un * ux) / dfac
    py = (ny + g * b[1] + (g - 1.0) * un * uy) / dfac
    c = np.asarray(chi, np.float32).astype(np.float64)
    norm = np.maximum(np.abs(px), np.abs(py)) if cheb else 1.0
    ax = np.where(ok, px * c / norm, dx)
    ay = np.where(ok, py * c / norm, dy)
    return ax, ay, np.where(ok, np.log(dfac), 0.0)
