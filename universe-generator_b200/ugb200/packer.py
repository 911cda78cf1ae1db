"""Python host side of the packer: universes, batches and results.

``Universe`` mirrors one reference engine run (the flags of
cuda/braid_cuda.cu:534-584 / cuda/braid_cuda3d.cu:862-913); ``Packer`` runs a
batch of them on one GPU through libug.so and returns the accepted set, the
trajectories and the worldline parameters.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


@dataclass
class Universe:
    dim: int = 2
    T: int = 64
    terms: int = 0                 # sinusoid terms per axis incl. sin1; 0 = full band
    rng: int = L.RNG_PHILOX
    zgrid: int = L.ZGRID_REF
    excl: int = L.EXCL_REF
    cross1d: int = 0
    pin_sin1: int = 0
    group_mode: int = L.GROUP_NONE
    round_size: int = 0            # candidates per round (0 = 65536); results do not depend on it
    seed: int = 0
    attempts: int = 100_000
    max_n: int = 0
    sub_attempts: int = 0
    accept_rate: float = 0.0
    sub_accept_rate: float = 0.0
    sub_fill_rate: float = 0.0     # --sub-until-fill-rate (newly occupied cells per attempt)
    euclid: int = 0                # --euclid-collision: L2 ball instead of the Chebyshev cube
    surv_cap: int = 0              # survivors resolved per round (0 = default); results do not depend on it

    @property
    def nw(self) -> int:
        return (self.terms or self.T) - 1

    def _c(self) -> L.UniverseCfg:
        return L.UniverseCfg(self.dim, self.T, self.terms, self.rng, self.zgrid, self.excl,
                             self.cross1d, self.pin_sin1, self.group_mode, self.round_size,
                             self.seed & (2**64 - 1), int(self.attempts), int(self.max_n),
                             int(self.sub_attempts), float(self.accept_rate),
                             float(self.sub_accept_rate), float(self.sub_fill_rate),
                             int(self.euclid), int(self.surv_cap))


@dataclass
class Stats:
    n: int
    n_unique: int
    n_sub: int
    attempts: int
    phase1_end: int
    rounds: int
    gray: int
    evals: int
    evals_fp64: int
    done: bool
    grid: str
    filled: int = 0              # occupied (timestep, cell) buckets of the collision grid
    visits: int = 0              # accepted points examined by the prefilter's neighbour tests


@dataclass
class Packer:
    universes: list[Universe]
    precision: int = L.PREC_FP64
    device: int = -1
    rounds_per_sync: int = 8
    use_graph: bool = True
    kernel_timing: bool = False
    stream: int = 0
    slot_hint: int = 0
    force_hash: bool = False
    _h: C.c_void_p = field(default=None, init=False, repr=False)

    def __post_init__(self) -> None:
        lib = L.load()
        n = len(self.universes)
        arr = (L.UniverseCfg * n)(*[u._c() for u in self.universes])
        opts = L.RunOpts(self.precision, self.device, self.rounds_per_sync,
                         int(self.use_graph), int(self.kernel_timing), int(self.force_hash),
                         self.stream,
                         self.slot_hint)
        h = C.c_void_p()
        L.check(lib.ug_batch_create(arr, n, C.byref(opts), C.byref(h)))
        self._h = h

    # -- running
    def run(self, max_rounds: int = 0) -> "Packer":
        L.check(L.load().ug_batch_run(self._h, max_rounds))
        return self

    def reset(self, seeds=None) -> "Packer":
        """Restart all universes from empty packings (optionally with new seeds)."""
        arr = None
        if seeds is not None:
            arr = np.ascontiguousarray(np.asarray(seeds, dtype=np.uint64))
            for u, s in zip(self.universes, arr):
                u.seed = int(s)
        L.check(L.load().ug_batch_reset(self._h, None if arr is None else arr.ctypes.data))
        return self

    def done(self) -> bool:
        rc = L.load().ug_batch_done(self._h)
        if rc < 0:
            raise L.UgError(-rc, L.last_error())
        return bool(rc)

    # -- results
    def stats(self, u: int = 0) -> Stats:
        s = L.Stats()
        L.check(L.load().ug_batch_stats(self._h, u, C.byref(s)))
        return Stats(s.n, s.n_unique, s.n_sub, s.attempts, s.phase1_end, s.rounds, s.gray,
                     s.evals, s.evals_fp64, s.state == 1, "hash" if s.grid_kind else "dense",
                     s.filled, s.visits)

    def accepted(self, u: int = 0) -> tuple[np.ndarray, np.ndarray]:
        lib = L.load()
        n = C.c_int64()
        L.check(lib.ug_batch_accepted(self._h, u, None, None, 0, C.byref(n)))
        idx = np.zeros(n.value, np.int64)
        gid = np.zeros(n.value, np.int32)
        if n.value:
            L.check(lib.ug_batch_accepted(self._h, u, idx.ctypes.data, gid.ctypes.data,
                                          n.value, C.byref(n)))
        return idx, gid

    def accepted_all(self) -> list[tuple[np.ndarray, np.ndarray]]:
        """(indices, group ids) of every universe, read back in one gather and one
        copy per array."""
        lib = L.load()
        n = len(self.universes)
        counts = np.zeros(n, np.int64)
        L.check(lib.ug_batch_accepted_all(self._h, None, None, 0, counts.ctypes.data))
        total = int(counts.sum())
        idx = np.zeros(total, np.int64)
        gid = np.zeros(total, np.int32)
        if total:
            L.check(lib.ug_batch_accepted_all(self._h, idx.ctypes.data, gid.ctypes.data, total,
                                              counts.ctypes.data))
        cuts = np.cumsum(counts)[:-1]
        return list(zip(np.split(idx, cuts), np.split(gid, cuts)))

    def positions(self, u: int = 0) -> np.ndarray:
        n = self.stats(u).n
        uni = self.universes[u]
        out = np.zeros((n, uni.dim, uni.T))
        L.check(L.load().ug_batch_positions(self._h, u, out.ctypes.data, n))
        return out

    def params(self, u: int = 0) -> dict:
        n = self.stats(u).n
        uni = self.universes[u]
        d, nw = uni.dim, uni.nw
        a2 = np.zeros((n, d))
        a = np.zeros((n, d, nw))
        f = np.zeros((n, d, nw))
        b = np.zeros((n, d, nw), np.int32)
        L.check(L.load().ug_batch_params(self._h, u, a2.ctypes.data, a.ctypes.data,
                                         b.ctypes.data, f.ctypes.data, n))
        return {"a2": a2, "a": a, "b": b, "f": f}

    def kernel_times(self) -> dict[str, tuple[float, int]]:
        kt = L.KernelTimes()
        L.check(L.load().ug_batch_kernel_times(self._h, C.byref(kt)))
        out = {}
        for i in range(12):
            name = kt.names[i]
            if name:
                out[name.decode()] = (kt.ms[i], kt.launches[i])
        return out

    def counters(self) -> tuple[int, int, int]:
        """(kernel launches, host->device bytes, device->host bytes) so far."""
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        L.check(L.load().ug_batch_counters(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def reset_times(self) -> None:
        L.check(L.load().ug_batch_reset_times(self._h))

    def mixed_error(self, u: int = 0, first: int = 0, count: int = 4096) -> tuple[float, float, float]:
        """(max |X_mixed - X_fp64|, widest guard band, max error / own guard band)."""
        e = C.c_double()
        m = C.c_double()
        q = C.c_double()
        L.check(L.load().ug_batch_mixed_error(self._h, u, first, count, C.byref(e), C.byref(m),
                                              C.byref(q)))
        return e.value, m.value, q.value

    def probe(self, u: int = 0, n: int = 5_000_000, bins: int = 50,
              seed: int | None = None) -> tuple[np.ndarray, np.ndarray]:
        """--diag probe: (proposed, accepted) per x-centre bin of n fresh candidates
        tested against the packing as it stands (braid_cuda3d.cu:1645-1667).  The
        default stream is keyed by seed ^ 0xABCDEF1234567890, as the reference keys
        its probe generator."""
        if seed is None:
            seed = (self.universes[u].seed ^ 0xABCDEF1234567890) & (2**64 - 1)
        prop = np.zeros(bins, np.int64)
        acc = np.zeros(bins, np.int64)
        L.check(L.load().ug_batch_probe(self._h, u, seed, int(n), bins, prop.ctypes.data,
                                        acc.ctypes.data))
        return prop, acc

    # -- checkpoint / resume
    def checkpoint(self, u: int = 0) -> dict:
        """Everything needed to resume universe u: admissions (candidate indices in
        admission order, groups) and the opaque state block."""
        lib = L.load()
        idx, gid = self.accepted(u)
        state = (C.c_uint8 * int(lib.ug_state_bytes()))()
        L.check(lib.ug_batch_save_state(self._h, u, state))
        return {"idx": np.ascontiguousarray(idx, np.int64), "gid": np.ascontiguousarray(gid, np.int32),
                "state": bytes(state)}

    def restore(self, u: int, ck: dict) -> "Packer":
        """Rebuild universe u from a checkpoint of a universe of the same model and
        seed; run() then continues where the checkpointed run stopped."""
        lib = L.load()
        idx = np.ascontiguousarray(ck["idx"], np.int64)
        gid = np.ascontiguousarray(ck["gid"], np.int32)
        state = C.create_string_buffer(bytes(ck["state"]), len(ck["state"]))
        L.check(lib.ug_batch_restore(self._h, u, len(idx), idx.ctypes.data, gid.ctypes.data, state))
        return self

    def close(self) -> None:
        if self._h:
            L.load().ug_batch_destroy(self._h)
            self._h = None

    def __enter__(self) -> "Packer":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


def save_checkpoint(path, ck: dict) -> None:
    np.savez(path, idx=ck["idx"], gid=ck["gid"], state=np.frombuffer(ck["state"], np.uint8))


def load_checkpoint(path) -> dict:
    z = np.load(path)
    return {"idx": z["idx"], "gid": z["gid"], "state": z["state"].tobytes()}


def pack(universe: Universe, precision: int = L.PREC_FP64, **kw):
    """Run one universe to its stop rule; returns (stats, accepted idx, gid)."""
    with Packer([universe], precision=precision, **kw) as p:
        p.run()
        idx, gid = p.accepted(0)
        return p.stats(0), idx, gid
